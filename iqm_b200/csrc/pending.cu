// Entry points whose kernels are not written yet: they fail loudly with IQM_EUNSUPPORTED.
#include "iqm_internal.cuh"

#define IQM_PENDING(name) throw iqm::Error{IQM_EUNSUPPORTED, name " is not implemented in this build"}
#define IQM_API extern "C" __attribute__((visibility("default")))

IQM_API void iqm_flip_default_params(iqm_flip_params *p) {
    if (!p) return;
    p->monitor_resolution_x = 2560.f;
    p->monitor_distance = 0.7f;
    p->monitor_width = 0.6f;
}
IQM_API double iqm_flip_ppd(const iqm_flip_params *) { return 0; }
IQM_API int iqm_flip(iqm_ctx *ctx, const uint8_t *, const uint8_t *, int, int, size_t, const iqm_flip_params *,
                     float *, double *) {
    return iqm::guarded(ctx, [&] { IQM_PENDING("iqm_flip"); });
}
IQM_API int iqm_flip_dev(iqm_ctx *ctx, const iqm_pair *, int, const iqm_flip_params *, double *) {
    return iqm::guarded(ctx, [&] { IQM_PENDING("iqm_flip_dev"); });
}
IQM_API int iqm_flip_batch(iqm_ctx *ctx, const iqm_pair *, int, const iqm_flip_params *, double *) {
    return iqm::guarded(ctx, [&] { IQM_PENDING("iqm_flip_batch"); });
}
