// Internal declarations shared by the library's translation units (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "iqm_cuda.h"

namespace iqm {

// Failure carried from deep inside an entry point to its C-ABI wrapper.
struct Error {
    int code;
    std::string msg;
};

#define IQM_CHECK_CUDA(expr)                                                              \
    do {                                                                                  \
        cudaError_t e_ = (expr);                                                          \
        if (e_ != cudaSuccess)                                                            \
            throw ::iqm::Error{IQM_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

#define IQM_REQUIRE(cond, text)                                   \
    do {                                                          \
        if (!(cond)) throw ::iqm::Error{IQM_EINVAL, (text)};      \
    } while (0)

// Grow-only device buffer: reused across calls, reallocated (after a stream sync) only when a
// request exceeds its capacity.
struct DevBuf {
    void *ptr = nullptr;
    size_t cap = 0;
    void *get(size_t bytes, cudaStream_t s) {
        if (bytes <= cap) return ptr;
        if (ptr) {
            IQM_CHECK_CUDA(cudaStreamSynchronize(s));
            cudaFree(ptr);
            ptr = nullptr;
            cap = 0;
        }
        size_t want = bytes < 4096 ? 4096 : bytes;
        want = (want + 255) & ~size_t(255);
        if (cudaMalloc(&ptr, want) != cudaSuccess) {
            cudaGetLastError();
            throw Error{IQM_ENOMEM, "device allocation of " + std::to_string(want) + " bytes failed"};
        }
        cap = want;
        return ptr;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
    }
};

// Pinned host staging buffer (grow-only), for small descriptor uploads and score readback.
struct PinnedBuf {
    void *ptr = nullptr;
    size_t cap = 0;
    void *get(size_t bytes, cudaStream_t s) {
        if (bytes <= cap) return ptr;
        if (ptr) {
            IQM_CHECK_CUDA(cudaStreamSynchronize(s));
            cudaFreeHost(ptr);
            ptr = nullptr;
            cap = 0;
        }
        size_t want = bytes < 4096 ? 4096 : bytes;
        if (cudaMallocHost(&ptr, want) != cudaSuccess) {
            cudaGetLastError();
            throw Error{IQM_ENOMEM, "pinned host allocation failed"};
        }
        cap = want;
        return ptr;
    }
    void release() {
        if (ptr) cudaFreeHost(ptr);
        ptr = nullptr;
        cap = 0;
    }
};

// Small host->device uploads (descriptors, parameters) through a ring of pinned slots.  Each slot
// is reused only after the event recorded behind its copy has completed, so callers never block
// on the stream and never overwrite bytes a pending copy still reads.
struct UploadRing {
    static constexpr int SLOTS = 8;
    void *host[SLOTS] = {};
    size_t cap[SLOTS] = {};
    cudaEvent_t ev[SLOTS] = {};
    int next = 0;
    void release() {
        for (int i = 0; i < SLOTS; i++) {
            if (ev[i]) cudaEventDestroy(ev[i]);
            if (host[i]) cudaFreeHost(host[i]);
            ev[i] = nullptr;
            host[i] = nullptr;
            cap[i] = 0;
        }
    }
};

// Launch-shape choices of the FSIM transform passes (0 / -1 = built-in heuristic).  They change
// only how work is split over CTAs, never a result bit; batch plans autotune them (plan.cu).
struct FsimTune {
    int chunk_mb = 0;     // L2 budget for the inverse-pass intermediates of one chunk of pairs
    int icols_lw = -1;    // log2 warps per CTA of the inverse column pass (clamped to what fits)
    int rows_per_cta = 0; // rows per CTA of the inverse row pass (1 or 2, if it fits)
};

struct FsimPlan;  // per plane-size FSIM constants (fsim.cu)
struct FftPlan;   // per-length FFT tables (fft.cu)

}  // namespace iqm

struct iqm_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string last_error;
    int launches = 0;  // kernel launches enqueued by the last entry point
    bool capturing = false;  // a batch plan is capturing the stream into a CUDA graph (plan.cu)
    iqm::FsimTune fsim_tune;
    // streams that independent work forks onto from `stream` and joins back from (iqm::side_streams)
    std::vector<cudaStream_t> side_streams;
    std::vector<cudaEvent_t> side_events;
    cudaEvent_t fork_event = nullptr;
    std::vector<cudaEvent_t> aux_events;  // further fork points (iqm::aux_event)
    // host-image uploads of the batch entry points run on their own stream, chunk by chunk, so a
    // chunk's copy overlaps the previous chunk's kernels (iqm::upload_pipelined)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copy_events[2] = {nullptr, nullptr};

    // named scratch areas (each grow-only)
    iqm::DevBuf desc;      // per-call pair descriptors
    iqm::DevBuf scratch;   // per-call kernel scratch (partials, counters, planes)
    iqm::DevBuf images;    // device copies of host images (host entry points)
    iqm::DevBuf maps;      // device map outputs (host entry points)
    iqm::DevBuf scores;    // device scores (host entry points)
    iqm::PinnedBuf pinned; // staging
    iqm::UploadRing ring;  // small async uploads

    std::map<std::pair<int, int>, iqm::FsimPlan *> fsim_plans;  // owned; freed by iqm_release_fsim_plans
    std::map<int, iqm::FftPlan *> fft_plans;  // owned; freed by iqm_release_fft_plans

    // Per-kernel device timing (iqm_set_kernel_timing): an event after every launch and after every
    // copy or memset the context enqueues; a kernel is charged the interval since the event before it.
    bool timing = false;
    std::vector<std::pair<const char *, cudaEvent_t>> marks;  // nullptr name: not a kernel
    std::vector<cudaEvent_t> event_pool;
    std::map<std::string, std::pair<long, double>> kernel_ms;  // name -> (launches, total ms)
};

namespace iqm {

// Records a timing event on the context stream when per-kernel timing is on (ctx.cu); `kernel` is
// the kernel launched just before, or nullptr after a copy, memset or call start.
void timing_mark(iqm_ctx *ctx, const char *kernel);

// Run `fn` and convert any failure into a status code recorded on the context.
template <class F>
int guarded(iqm_ctx *ctx, F &&fn) {
    if (!ctx) return IQM_EINVAL;
    try {
        ctx->launches = 0;
        IQM_CHECK_CUDA(cudaSetDevice(ctx->device));
        timing_mark(ctx, nullptr);
        fn();
        ctx->last_error.clear();
        return IQM_OK;
    } catch (const Error &e) {
        ctx->last_error = e.msg;
        return e.code;
    } catch (const std::bad_alloc &) {
        ctx->last_error = "host allocation failed";
        return IQM_ENOMEM;
    } catch (const std::exception &e) {
        ctx->last_error = e.what();
        return IQM_EINVAL;
    }
}

inline void check_launch(iqm_ctx *ctx, const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw Error{IQM_ECUDA, std::string(what) + ": " + cudaGetErrorString(e)};
    ctx->launches++;
    timing_mark(ctx, what);
}

// Validate a batch of pair descriptors.
inline void check_pairs(const iqm_pair *pairs, int n, int min_w, int min_h) {
    IQM_REQUIRE(pairs != nullptr, "pairs is NULL");
    IQM_REQUIRE(n >= 1, "pair count must be >= 1");
    for (int i = 0; i < n; i++) {
        const iqm_pair &p = pairs[i];
        IQM_REQUIRE(p.input && p.ref, "pair " + std::to_string(i) + ": image pointer is NULL");
        IQM_REQUIRE(p.w >= min_w && p.h >= min_h,
                    "pair " + std::to_string(i) + ": image too small (" + std::to_string(p.w) + "x" +
                        std::to_string(p.h) + ")");
        IQM_REQUIRE(p.w <= 65536 && p.h <= 65536 && (long long)p.w * p.h < (1LL << 31),
                    "pair " + std::to_string(i) + ": image too large (at most 65536 per side and 2^31 pixels)");
        IQM_REQUIRE(p.row_bytes >= size_t(p.w) * 4, "pair " + std::to_string(i) + ": row_bytes < 4*w");
    }
}

// Device-resident pairs are read in place with 4-byte pixel loads (and wider ones when the base and
// pitch allow), so both image pointers and the pitch must be multiples of 4; anything else is
// rejected here instead of faulting on the GPU.  Host entry points repack into aligned buffers.
inline void check_dev_alignment(const iqm_pair *pairs, int n) {
    for (int i = 0; i < n; i++) {
        const iqm_pair &p = pairs[i];
        IQM_REQUIRE(((reinterpret_cast<uintptr_t>(p.input) | reinterpret_cast<uintptr_t>(p.ref) |
                      uintptr_t(p.row_bytes)) & 3u) == 0,
                    "pair " + std::to_string(i) + ": device image pointers and row_bytes must be multiples of 4");
    }
}

// Copies `bytes` from host memory to `dst` (grown as needed) on the context stream, staging
// through the pinned ring; returns the device pointer.
void *upload_bytes(iqm_ctx *ctx, DevBuf &dst, const void *src, size_t bytes);

// Makes at least n side streams (with one join event each) and the fork event exist on the context.
void side_streams(iqm_ctx *ctx, int n);
// Event i of the context's auxiliary pool (created on first use; timing disabled).
cudaEvent_t aux_event(iqm_ctx *ctx, int i);

// Copies host pairs to device memory (inside ctx->images) and rewrites the pointers.
std::vector<iqm_pair> upload_pairs(iqm_ctx *ctx, const iqm_pair *pairs, int n);

// Copies host pairs to device memory in chunks of whole pairs on the context's copy stream and,
// as each chunk lands, calls run(dev, first, count) to enqueue that chunk's work on the context
// stream (dev: the chunk's device descriptors; first: its index in `pairs`): chunk k + 1's copy
// overlaps chunk k's kernels.  Per-kernel timing keeps everything on the context stream.
void upload_pipelined(iqm_ctx *ctx, const iqm_pair *pairs, int n,
                      const std::function<void(const iqm_pair *dev, int first, int count)> &run);

// Validate and enqueue one metric for device-resident pairs on the context stream (the bodies of
// the iqm_*_dev entry points); batch plans call them directly.
void enqueue_ssim_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n, const iqm_ssim_params *params, double *d_scores);
void enqueue_fsim_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n, iqm_precision precision, int energy_mode,
                      double *d_scores);
void enqueue_flip_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n, const iqm_flip_params *params, double *d_scores);
void enqueue_msvd_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n, double *d_scores);

inline unsigned ceil_div(long a, long b) { return unsigned((a + b - 1) / b); }

// Per-pixel transcendentals from the SFU approximations (a few ulp, far inside the 1e-5 score
// bounds; the reference's shaders leave the accuracy of sqrt, pow and division to the implementation
// as well).  The PTX .ftz forms are single SFU operations.  Flushing subnormals changes nothing for
// the kernels' arguments: square roots and reciprocals get clamped or bounded-below values, and the
// bases of the powers (colour and feature differences, products of similarity ratios) are either
// exactly 0 or at least an ulp of their FP32 operands, far above the subnormal range.
#ifdef __CUDACC__
__device__ __forceinline__ float ex2_approx(float x) {  // 2^x
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float lg2_approx(float x) {  // log2 x (-inf for 0)
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rsqrt_approx(float x) {  // 1 / sqrt(x)
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {  // 1 / x
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// sqrt(v) for v >= 0 as v * rsqrt(v); 0 for v = 0
__device__ __forceinline__ float sqrt_nonneg(float v) { return v * rsqrt_approx(fmaxf(v, 1e-30f)); }
// x^y for x >= 0: exp2(y log2 x) for x > 0; for x = 0 the values of pow(0, y): 0 for y > 0, 1 for
// y = 0, +inf for y < 0
__device__ __forceinline__ float pow_nonneg(float x, float y) {
    return x > 0.0f ? ex2_approx(y * lg2_approx(x)) : (y > 0.0f ? 0.0f : y == 0.0f ? 1.0f : __int_as_float(0x7f800000));
}
// cube root of a normal v > 0: exp2(log2(v) / 3), then one Newton-Raphson step on y^3 = v,
// y <- y - (y^3 - v) / (3 y^2), which squares the estimate's relative error
__device__ __forceinline__ float cbrt_pos(float v) {
    const float y = ex2_approx(lg2_approx(v) * (1.0f / 3.0f));
    const float y2 = y * y;
    return y - fmaf(y2, y, -v) * rcp_approx(3.0f * y2);
}
#endif

}  // namespace iqm
