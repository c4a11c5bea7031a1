// Context management and shared host plumbing of the C ABI (include/iqm_cuda.h).
//
// Replaces the reference's VulkanRuntime (src/gpu/base/vulkan_runtime.{h,cpp}): device choice,
// one stream instead of the compute/transfer queues, and grow-only device buffers instead of the
// per-call buffer/image creation every computeMetric performs (e.g. src/gpu/ssim/ssim.cpp:245-384).
#include <cstring>

#include "iqm_internal.cuh"

namespace {
thread_local std::string g_create_error;
}

extern "C" __attribute__((visibility("default"))) int iqm_create(int device, iqm_ctx **out) {
    if (!out) return IQM_EINVAL;
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) {
        g_create_error = std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e);
        return IQM_ECUDA;
    }
    if (device < 0 || device >= count) {
        g_create_error = "device index " + std::to_string(device) + " out of range (" +
                         std::to_string(count) + " devices)";
        return IQM_EINVAL;
    }
    e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        g_create_error = std::string("cudaSetDevice: ") + cudaGetErrorString(e);
        return IQM_ECUDA;
    }
    auto *ctx = new (std::nothrow) iqm_ctx();
    if (!ctx) return IQM_ENOMEM;
    ctx->device = device;
    e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        g_create_error = std::string("cudaStreamCreate: ") + cudaGetErrorString(e);
        delete ctx;
        return IQM_ECUDA;
    }
    ctx->stream = ctx->own_stream;
    g_create_error.clear();
    *out = ctx;
    return IQM_OK;
}

void iqm_release_fsim_plans(iqm_ctx *ctx);  // fsim.cu
void iqm_release_fft_plans(iqm_ctx *ctx);   // fft.cu

extern "C" __attribute__((visibility("default"))) int iqm_destroy(iqm_ctx *ctx) {
    if (!ctx) return IQM_EINVAL;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    iqm_release_fsim_plans(ctx);
    iqm_release_fft_plans(ctx);
    ctx->desc.release();
    ctx->scratch.release();
    ctx->images.release();
    ctx->maps.release();
    ctx->scores.release();
    ctx->pinned.release();
    ctx->ring.release();
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return IQM_OK;
}

extern "C" __attribute__((visibility("default"))) const char *iqm_last_error(const iqm_ctx *ctx) {
    return ctx ? ctx->last_error.c_str() : g_create_error.c_str();
}

extern "C" __attribute__((visibility("default"))) int iqm_set_stream(iqm_ctx *ctx, void *cuda_stream) {
    // The context's buffers are reused call after call in stream order; finish the work queued
    // on the previous stream before later calls can touch them from another stream.
    return iqm::guarded(ctx, [&] {
        IQM_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : ctx->own_stream;
    });
}

extern "C" __attribute__((visibility("default"))) int iqm_synchronize(iqm_ctx *ctx) {
    return iqm::guarded(ctx, [&] { IQM_CHECK_CUDA(cudaStreamSynchronize(ctx->stream)); });
}

extern "C" __attribute__((visibility("default"))) int iqm_device_name(iqm_ctx *ctx, char *buf, size_t len) {
    return iqm::guarded(ctx, [&] {
        IQM_REQUIRE(buf && len > 0, "buffer is NULL");
        cudaDeviceProp prop;
        IQM_CHECK_CUDA(cudaGetDeviceProperties(&prop, ctx->device));
        std::snprintf(buf, len, "%s", prop.name);
    });
}

extern "C" __attribute__((visibility("default"))) int iqm_last_launch_count(const iqm_ctx *ctx) { return ctx ? ctx->launches : 0; }

namespace iqm {

void *upload_bytes(iqm_ctx *ctx, DevBuf &dst, const void *src, size_t bytes) {
    UploadRing &r = ctx->ring;
    const int slot = r.next;
    r.next = (r.next + 1) % UploadRing::SLOTS;
    if (r.ev[slot]) {
        IQM_CHECK_CUDA(cudaEventSynchronize(r.ev[slot]));
    } else {
        IQM_CHECK_CUDA(cudaEventCreateWithFlags(&r.ev[slot], cudaEventDisableTiming));
    }
    if (r.cap[slot] < bytes) {
        if (r.host[slot]) cudaFreeHost(r.host[slot]);
        r.host[slot] = nullptr;
        r.cap[slot] = 0;
        size_t want = bytes < 4096 ? 4096 : bytes;
        if (cudaMallocHost(&r.host[slot], want) != cudaSuccess) {
            cudaGetLastError();
            throw Error{IQM_ENOMEM, "pinned host allocation failed"};
        }
        r.cap[slot] = want;
    }
    std::memcpy(r.host[slot], src, bytes);
    void *d = dst.get(bytes, ctx->stream);
    IQM_CHECK_CUDA(cudaMemcpyAsync(d, r.host[slot], bytes, cudaMemcpyHostToDevice, ctx->stream));
    IQM_CHECK_CUDA(cudaEventRecord(r.ev[slot], ctx->stream));
    return d;
}

std::vector<iqm_pair> upload_pairs(iqm_ctx *ctx, const iqm_pair *pairs, int n) {
    // Device copies use a 16-byte-aligned pitch so kernels can take their vector-load path.
    std::vector<iqm_pair> dev(pairs, pairs + n);
    std::vector<size_t> offs(n);
    size_t total = 0;
    for (int i = 0; i < n; i++) {
        size_t pitch = (size_t(pairs[i].w) * 4 + 15) & ~size_t(15);
        size_t bytes = (pitch * size_t(pairs[i].h) + 255) & ~size_t(255);
        offs[i] = total;
        total += 2 * bytes;
        dev[i].row_bytes = pitch;
    }
    auto *base = static_cast<uint8_t *>(ctx->images.get(total, ctx->stream));
    for (int i = 0; i < n; i++) {
        size_t pitch = dev[i].row_bytes;
        size_t bytes = (pitch * size_t(pairs[i].h) + 255) & ~size_t(255);
        uint8_t *din = base + offs[i], *dref = base + offs[i] + bytes;
        IQM_CHECK_CUDA(cudaMemcpy2DAsync(din, pitch, pairs[i].input, pairs[i].row_bytes,
                                         size_t(pairs[i].w) * 4, pairs[i].h, cudaMemcpyHostToDevice,
                                         ctx->stream));
        IQM_CHECK_CUDA(cudaMemcpy2DAsync(dref, pitch, pairs[i].ref, pairs[i].row_bytes,
                                         size_t(pairs[i].w) * 4, pairs[i].h, cudaMemcpyHostToDevice,
                                         ctx->stream));
        dev[i].input = din;
        dev[i].ref = dref;
    }
    return dev;
}

}  // namespace iqm
