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

namespace iqm {
static void timing_release(iqm_ctx *ctx);
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
    iqm::timing_release(ctx);
    for (auto st : ctx->side_streams) cudaStreamDestroy(st);
    for (auto ev : ctx->side_events) cudaEventDestroy(ev);
    for (auto ev : ctx->aux_events) cudaEventDestroy(ev);
    if (ctx->fork_event) cudaEventDestroy(ctx->fork_event);
    if (ctx->copy_stream) {
        cudaStreamSynchronize(ctx->copy_stream);
        cudaStreamDestroy(ctx->copy_stream);
    }
    for (auto ev : ctx->copy_events)
        if (ev) cudaEventDestroy(ev);
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

extern "C" __attribute__((visibility("default"))) int iqm_host_alloc(size_t bytes, void **out) {
    if (!out) return IQM_EINVAL;
    *out = nullptr;
    if (bytes == 0) return IQM_EINVAL;
    if (cudaMallocHost(out, bytes) != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return IQM_ENOMEM;
    }
    return IQM_OK;
}

extern "C" __attribute__((visibility("default"))) int iqm_host_free(void *p) {
    if (!p) return IQM_OK;
    return cudaFreeHost(p) == cudaSuccess ? IQM_OK : IQM_ECUDA;
}

namespace iqm {

void *upload_bytes(iqm_ctx *ctx, DevBuf &dst, const void *src, size_t bytes) {
    if (ctx->capturing) {
        // A batch plan captures a second, identical enqueue: the bytes are already on the device
        // (uploaded by the uncaptured pass into the plan's own buffer) and a copy node would read a
        // staging slot that later calls reuse.
        (void)src;
        IQM_REQUIRE(dst.ptr && bytes <= dst.cap, "batch plan capture: descriptor buffer not prepared");
        return dst.ptr;
    }
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
    timing_mark(ctx, nullptr);
    return d;
}

void side_streams(iqm_ctx *ctx, int n) {
    if (!ctx->fork_event) IQM_CHECK_CUDA(cudaEventCreateWithFlags(&ctx->fork_event, cudaEventDisableTiming));
    while (int(ctx->side_streams.size()) < n) {
        cudaStream_t st = nullptr;
        cudaEvent_t ev = nullptr;
        IQM_CHECK_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaStreamDestroy(st);
            throw Error{IQM_ECUDA, "cudaEventCreate failed"};
        }
        ctx->side_streams.push_back(st);
        ctx->side_events.push_back(ev);
    }
}

cudaEvent_t aux_event(iqm_ctx *ctx, int i) {
    while (int(ctx->aux_events.size()) <= i) {
        cudaEvent_t ev = nullptr;
        IQM_CHECK_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        ctx->aux_events.push_back(ev);
    }
    return ctx->aux_events[i];
}

// Device layout of host pairs in ctx->images: a 16-byte-aligned pitch per image (so kernels can
// take their vector-load path); returns the descriptors with device pointers.
static std::vector<iqm_pair> device_layout(iqm_ctx *ctx, const iqm_pair *pairs, int n) {
    std::vector<iqm_pair> dev(pairs, pairs + n);
    std::vector<size_t> offs(n);
    size_t total = 0;
    for (int i = 0; i < n; i++) {
        const size_t pitch = (size_t(pairs[i].w) * 4 + 15) & ~size_t(15);
        const size_t bytes = (pitch * size_t(pairs[i].h) + 255) & ~size_t(255);
        offs[i] = total;
        total += 2 * bytes;
        dev[i].row_bytes = pitch;
    }
    auto *base = static_cast<uint8_t *>(ctx->images.get(total, ctx->stream));
    for (int i = 0; i < n; i++) {
        const size_t bytes = (dev[i].row_bytes * size_t(pairs[i].h) + 255) & ~size_t(255);
        dev[i].input = base + offs[i];
        dev[i].ref = base + offs[i] + bytes;
    }
    return dev;
}

// Copies one image: a single linear copy when both pitches equal the row, else a 2-D copy.
static void copy_image(const uint8_t *dst, size_t dpitch, const uint8_t *src, size_t spitch, int w, int h,
                       cudaStream_t st) {
    const size_t row = size_t(w) * 4;
    void *d = const_cast<uint8_t *>(dst);
    if (spitch == row && dpitch == row) {
        IQM_CHECK_CUDA(cudaMemcpyAsync(d, src, row * size_t(h), cudaMemcpyHostToDevice, st));
    } else {
        IQM_CHECK_CUDA(cudaMemcpy2DAsync(d, dpitch, src, spitch, row, h, cudaMemcpyHostToDevice, st));
    }
}

std::vector<iqm_pair> upload_pairs(iqm_ctx *ctx, const iqm_pair *pairs, int n) {
    std::vector<iqm_pair> dev = device_layout(ctx, pairs, n);
    for (int i = 0; i < n; i++) {
        copy_image(dev[i].input, dev[i].row_bytes, pairs[i].input, pairs[i].row_bytes, pairs[i].w, pairs[i].h,
                   ctx->stream);
        copy_image(dev[i].ref, dev[i].row_bytes, pairs[i].ref, pairs[i].row_bytes, pairs[i].w, pairs[i].h, ctx->stream);
    }
    timing_mark(ctx, nullptr);
    return dev;
}

void upload_pipelined(iqm_ctx *ctx, const iqm_pair *pairs, int n,
                      const std::function<void(const iqm_pair *dev, int first, int count)> &run) {
    std::vector<iqm_pair> dev = device_layout(ctx, pairs, n);
    size_t total = 0;
    for (int i = 0; i < n; i++) total += 2 * dev[i].row_bytes * size_t(pairs[i].h);
    // about eight chunks of whole pairs, none below 32 MB of images (a chunk's kernels then run
    // long enough to cover the start of the next copy)
    constexpr size_t kMinChunk = size_t(32) << 20;
    const size_t target = std::max(kMinChunk, total / 8);
    const bool overlap = !ctx->timing && total > target;
    cudaStream_t cs = ctx->stream;
    if (overlap) {
        if (!ctx->copy_stream) IQM_CHECK_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
        for (auto &ev : ctx->copy_events)
            if (!ev) IQM_CHECK_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        cs = ctx->copy_stream;
        // work already enqueued on the context stream may still read the image buffer
        IQM_CHECK_CUDA(cudaEventRecord(ctx->copy_events[0], ctx->stream));
        IQM_CHECK_CUDA(cudaStreamWaitEvent(cs, ctx->copy_events[0], 0));
    }
    for (int first = 0; first < n;) {
        int last = first;
        size_t bytes = 0;
        do {
            bytes += 2 * dev[last].row_bytes * size_t(pairs[last].h);
            last++;
        } while (last < n && bytes < target);
        for (int i = first; i < last; i++) {
            copy_image(dev[i].input, dev[i].row_bytes, pairs[i].input, pairs[i].row_bytes, pairs[i].w, pairs[i].h, cs);
            copy_image(dev[i].ref, dev[i].row_bytes, pairs[i].ref, pairs[i].row_bytes, pairs[i].w, pairs[i].h, cs);
        }
        if (overlap) {
            // a wait takes the event's state at the time of the call, so one event serves every chunk
            IQM_CHECK_CUDA(cudaEventRecord(ctx->copy_events[1], cs));
            IQM_CHECK_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->copy_events[1], 0));
        }
        timing_mark(ctx, nullptr);
        run(dev.data() + first, first, last - first);
        first = last;
    }
}

// Charges every kernel mark the interval since the mark before it, then recycles the events.
// Waits for the context stream.
static void timing_collect(iqm_ctx *ctx) {
    if (ctx->marks.empty()) return;
    IQM_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    for (size_t i = 1; i < ctx->marks.size(); i++) {
        if (!ctx->marks[i].first) continue;
        float ms = 0.f;
        IQM_CHECK_CUDA(cudaEventElapsedTime(&ms, ctx->marks[i - 1].second, ctx->marks[i].second));
        auto &acc = ctx->kernel_ms[ctx->marks[i].first];
        acc.first++;
        acc.second += ms;
    }
    // the last mark starts the next interval
    auto last = ctx->marks.back();
    for (size_t i = 0; i + 1 < ctx->marks.size(); i++) ctx->event_pool.push_back(ctx->marks[i].second);
    ctx->marks.clear();
    ctx->marks.push_back({nullptr, last.second});
}

static void timing_release(iqm_ctx *ctx) {
    for (auto &m : ctx->marks) cudaEventDestroy(m.second);
    for (auto e : ctx->event_pool) cudaEventDestroy(e);
    ctx->marks.clear();
    ctx->event_pool.clear();
}

void timing_mark(iqm_ctx *ctx, const char *kernel) {
    if (!ctx->timing || ctx->capturing) return;
    // A stream switch or a long run: settle what is recorded so far (the settled mark stays the
    // start of the next interval).
    if (ctx->marks.size() >= 16384) timing_collect(ctx);
    cudaEvent_t ev;
    if (!ctx->event_pool.empty()) {
        ev = ctx->event_pool.back();
        ctx->event_pool.pop_back();
    } else {
        IQM_CHECK_CUDA(cudaEventCreate(&ev));
    }
    const cudaError_t e = cudaEventRecord(ev, ctx->stream);
    if (e != cudaSuccess) {
        ctx->event_pool.push_back(ev);
        throw Error{IQM_ECUDA, std::string("cudaEventRecord: ") + cudaGetErrorString(e)};
    }
    ctx->marks.push_back({kernel, ev});
}

}  // namespace iqm

extern "C" __attribute__((visibility("default"))) int iqm_set_kernel_timing(iqm_ctx *ctx, int enable) {
    return iqm::guarded(ctx, [&] {
        if (ctx->timing) iqm::timing_collect(ctx);
        iqm::timing_release(ctx);
        ctx->kernel_ms.clear();
        ctx->timing = enable != 0;
    });
}

extern "C" __attribute__((visibility("default"))) int iqm_kernel_times(iqm_ctx *ctx, char *buf, size_t cap) {
    return iqm::guarded(ctx, [&] {
        IQM_REQUIRE(buf && cap > 0, "buffer is NULL");
        iqm::timing_collect(ctx);
        std::string out;
        char line[256];
        for (const auto &kv : ctx->kernel_ms) {
            std::snprintf(line, sizeof(line), "%s %ld %.6f\n", kv.first.c_str(), kv.second.first, kv.second.second);
            out += line;
        }
        IQM_REQUIRE(out.size() < cap, "buffer too small for the kernel time report");
        std::memcpy(buf, out.c_str(), out.size() + 1);
    });
}
