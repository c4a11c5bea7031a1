#include "iqm_cuda.hpp"

#include <stdexcept>

namespace IQM::CUDA {

Runtime::Runtime(int device) {
    const int rc = iqm_create(device, &ctx);
    if (rc != IQM_OK) throw std::runtime_error(std::string("CUDA runtime: ") + iqm_last_error(nullptr));
    char name[256] = {0};
    check(iqm_device_name(ctx, name, sizeof(name)));
    selectedDevice = name;
}

Runtime::~Runtime() {
    if (ctx) iqm_destroy(ctx);
}

void Runtime::check(int rc) const {
    if (rc != IQM_OK) throw std::runtime_error(iqm_last_error(ctx));
}

SSIMResult SSIM::computeMetric(const Runtime &rt, const InputImage &image, const InputImage &ref) {
    SSIMResult res{std::vector<float>(size_t(image.width) * image.height), unsigned(image.width),
                   unsigned(image.height), 0.f, {}};
    const iqm_ssim_params p{kernelSize, k_1, k_2, sigma, int(precision)};
    double mssim = 0;
    res.timestamps.mark("start GPU pipeline");
    rt.check(iqm_ssim(rt.ctx, image.data.data(), ref.data.data(), image.width, image.height,
                      size_t(image.width) * 4, &p, res.imageData.data(), &mssim));
    res.mssim = float(mssim);
    res.timestamps.mark("MSSIM computed");
    return res;
}

SVDResult SVD::computeMetric(const Runtime &rt, const InputImage &image, const InputImage &ref) {
    SVDResult res{std::vector<float>(size_t(image.width / 8) * (image.height / 8)), unsigned(image.width / 8),
                  unsigned(image.height / 8), 0.f, {}};
    double msvd = 0;
    res.timestamps.mark("start GPU pipeline");
    rt.check(iqm_msvd(rt.ctx, image.data.data(), ref.data.data(), image.width, image.height,
                      size_t(image.width) * 4, res.imageData.data(), &msvd));
    res.msvd = float(msvd);
    res.timestamps.mark("M-SVD computed");
    return res;
}

FSIMResult FSIM::computeMetric(const Runtime &rt, const InputImage &image, const InputImage &ref) {
    FSIMResult res{0.f, 0.f, {}};
    double f = 0, fc = 0;
    res.timestamps.mark("start GPU pipeline");
    rt.check(iqm_fsim(rt.ctx, image.data.data(), ref.data.data(), image.width, image.height, size_t(image.width) * 4,
                      precision, energyMode, &f, &fc));
    res.fsim = float(f);
    res.fsimc = float(fc);
    res.timestamps.mark("FSIM, FSIMc computed");
    return res;
}

FLIPResult FLIP::computeMetric(const Runtime &rt, const InputImage &image, const InputImage &ref,
                               const FLIPArguments &args) {
    FLIPResult res{0.f, {}};
    const iqm_flip_params p{args.monitor_resolution_x, args.monitor_distance, args.monitor_width};
    double m = 0;
    if (wantMap) {
        res.imageData.resize(size_t(image.width) * image.height);
        res.width = unsigned(image.width);
        res.height = unsigned(image.height);
    }
    res.timestamps.mark("start GPU pipeline");
    rt.check(iqm_flip(rt.ctx, image.data.data(), ref.data.data(), image.width, image.height, size_t(image.width) * 4,
                      &p, wantMap ? res.imageData.data() : nullptr, &m));
    res.mean_flip = float(m);
    res.timestamps.mark("FLIP computed");
    return res;
}

}  // namespace IQM::CUDA
