// C++ classes with the reference's metric interface (src/gpu/{ssim,svd,fsim,flip}/*.h): one class
// per metric, constructed on a runtime, with computeMetric(runtime, image, ref[, args]) returning
// the reference's result structs by value.  They run on libiqm_cuda.so through include/iqm_cuda.h;
// failures are thrown as std::runtime_error, as the reference does.
#ifndef IQM_HOST_IQM_CUDA_HPP
#define IQM_HOST_IQM_CUDA_HPP

#include <string>
#include <vector>

#include "iqm_cuda.h"
#include "input_image.h"
#include "timestamps.h"

namespace IQM::CUDA {

// Stands in for IQM::GPU::VulkanRuntime (src/gpu/base/vulkan_runtime.h:15-82).
class Runtime {
public:
    explicit Runtime(int device = 0);
    ~Runtime();
    Runtime(const Runtime &) = delete;
    Runtime &operator=(const Runtime &) = delete;
    void check(int rc) const;
    iqm_ctx *ctx = nullptr;
    std::string selectedDevice;
};

struct SSIMResult {  // src/gpu/ssim/ssim.h:17-23
    std::vector<float> imageData;
    unsigned int width;
    unsigned int height;
    float mssim;
    Timestamps timestamps;
};

class SSIM {  // src/gpu/ssim/ssim.h:25-35
public:
    explicit SSIM(const Runtime &) {}
    SSIMResult computeMetric(const Runtime &runtime, const InputImage &image, const InputImage &ref);
    int kernelSize = 11;
    float k_1 = 0.01;
    float k_2 = 0.03;
    float sigma = 1.5;
    iqm_precision precision = IQM_FP32;  // IQM_MIXED / IQM_MIXED_FAST: tensor-core window sums
};

struct SVDResult {  // src/gpu/svd/svd.h:17-23
    std::vector<float> imageData;
    unsigned int width;
    unsigned int height;
    float msvd;
    Timestamps timestamps;
};

class SVD {  // src/gpu/svd/svd.h:25-28
public:
    explicit SVD(const Runtime &) {}
    SVDResult computeMetric(const Runtime &runtime, const InputImage &image, const InputImage &ref);
};

struct FSIMResult {  // src/gpu/fsim/fsim.h:27-31
    float fsim;
    float fsimc;
    Timestamps timestamps;
};

class FSIM {  // src/gpu/fsim/fsim.h:33-36
public:
    explicit FSIM(const Runtime &) {}
    FSIMResult computeMetric(const Runtime &runtime, const InputImage &image, const InputImage &ref);
    iqm_precision precision = IQM_FP32;
    int energyMode = 0;  // 0: noise-energy pooling as the reference (first ceil(N/2) pixels); 1: all N
};

struct FLIPResult {  // src/gpu/flip/flip.h:16-19; mean_flip is assigned here
    float mean_flip;
    Timestamps timestamps;
    // the per-pixel FLIP value (combine_error_maps.glsl:28), filled when FLIP::wantMap is set
    std::vector<float> imageData;
    unsigned int width = 0;
    unsigned int height = 0;
};

struct FLIPArguments {  // src/gpu/flip/flip.h:21-25
    float monitor_resolution_x = 2560;
    float monitor_distance = 0.7;
    float monitor_width = 0.6;
};

class FLIP {  // src/gpu/flip/flip.h:27-30
public:
    explicit FLIP(const Runtime &) {}
    FLIPResult computeMetric(const Runtime &runtime, const InputImage &image, const InputImage &ref,
                             const FLIPArguments &args);
    bool wantMap = false;
};

}  // namespace IQM::CUDA

#endif
