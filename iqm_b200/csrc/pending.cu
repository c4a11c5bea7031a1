// Entry points whose kernels are not written yet: they fail loudly with IQM_EUNSUPPORTED.
#include "iqm_internal.cuh"

namespace iqm { struct FsimPlan {}; struct FftPlan {}; }

#define IQM_PENDING(name) throw iqm::Error{IQM_EUNSUPPORTED, name " is not implemented in this build"}

void iqm_release_fsim_plans(iqm_ctx *ctx) { for (auto &kv : ctx->fsim_plans) delete kv.second; ctx->fsim_plans.clear(); }
void iqm_release_fft_plans(iqm_ctx *ctx) { for (auto &kv : ctx->fft_plans) delete kv.second; ctx->fft_plans.clear(); }

extern "C" __attribute__((visibility("default"))) void iqm_flip_default_params(iqm_flip_params *p) {
    if (!p) return;
    p->monitor_resolution_x = 2560.f;
    p->monitor_distance = 0.7f;
    p->monitor_width = 0.6f;
}
extern "C" __attribute__((visibility("default"))) double iqm_flip_ppd(const iqm_flip_params *p) { return 0; }
extern "C" __attribute__((visibility("default"))) int iqm_flip(iqm_ctx *ctx, const uint8_t *, const uint8_t *, int, int, size_t, const iqm_flip_params *, float *, double *) {
    return iqm::guarded(ctx, [&] { IQM_PENDING("iqm_flip"); });
}
extern "C" __attribute__((visibility("default"))) int iqm_fsim(iqm_ctx *ctx, const uint8_t *, const uint8_t *, int, int, size_t, iqm_precision, int, double *, double *) {
    return iqm::guarded(ctx, [&] { IQM_PENDING("iqm_fsim"); });
}
extern "C" __attribute__((visibility("default"))) int iqm_flip_dev(iqm_ctx *ctx, const iqm_pair *, int, const iqm_flip_params *, double *) { return iqm::guarded(ctx, [&] { IQM_PENDING("iqm_flip_dev"); }); }
extern "C" __attribute__((visibility("default"))) int iqm_fsim_dev(iqm_ctx *ctx, const iqm_pair *, int, iqm_precision, int, double *) { return iqm::guarded(ctx, [&] { IQM_PENDING("iqm_fsim_dev"); }); }
extern "C" __attribute__((visibility("default"))) int iqm_flip_batch(iqm_ctx *ctx, const iqm_pair *, int, const iqm_flip_params *, double *) { return iqm::guarded(ctx, [&] { IQM_PENDING("iqm_flip_batch"); }); }
extern "C" __attribute__((visibility("default"))) int iqm_fsim_batch(iqm_ctx *ctx, const iqm_pair *, int, iqm_precision, int, double *) { return iqm::guarded(ctx, [&] { IQM_PENDING("iqm_fsim_batch"); }); }
