// Command-line arguments with the reference's rules (src/args.h:15-24, src/args.cpp:9-61):
// `--method M --input A --ref B [--output P] [-v]`; every other `KEY VALUE` pair is kept in
// `options` (FLIP reads FLIP_WIDTH, FLIP_RES, FLIP_DISTANCE from there; the batch and repeat modes
// of this front end read --batch, --chunk, --threads, --repeat; FSIM and SSIM read --precision,
// FSIM reads FSIM_ENERGY_SUM).  A missing method, input or
// reference (input and reference are not needed with --batch), or an unknown method name, throws
// std::runtime_error.
#ifndef IQM_HOST_ARGS_H
#define IQM_HOST_ARGS_H

#include <optional>
#include <string>
#include <unordered_map>

#include "iqm_cuda.h"
#include "methods.h"

namespace IQM {
class Args {
public:
    Args(unsigned argc, const char *argv[]);
    Method method;
    std::string inputPath;
    std::string refPath;
    std::optional<std::string> outputPath;
    std::unordered_map<std::string, std::string> options;
    bool verbose = false;
};

// Options of this front end read from `options`: --precision fp32|mixed|mixed_fast (the form of
// FSIM and SSIM; default fp32) and FSIM_ENERGY_SUM reference|full (FSIM's noise-energy pooling; default
// reference).  Other values throw std::runtime_error.
iqm_precision precision_option(const Args &args);
int energy_option(const Args &args);
}  // namespace IQM

#endif
