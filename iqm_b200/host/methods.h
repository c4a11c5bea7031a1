// Metric selection, as the reference's src/methods.h:13-19 (same names and numbering).
#ifndef IQM_HOST_METHODS_H
#define IQM_HOST_METHODS_H

#include <string>

namespace IQM {
enum class Method {
    SSIM = 1,
    CW_SSIM_CPU = 2,
    SVD = 3,
    FSIM = 4,
    FLIP = 5,
};

// Display name (src/methods.cpp): "SSIM", "CW-SSIM", "SVD", "FSIM", "FLIP".
std::string method_name(const Method &method);
}  // namespace IQM

#endif
