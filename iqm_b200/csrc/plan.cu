// Batched evaluation: one call over many pairs and metrics (iqm_batch), and reusable batch plans
// (iqm_batch_plan_*) that autotune FSIM's launch shapes once and then replay the whole launch
// sequence of every requested metric as one CUDA graph.
//
// The reference evaluates one pair and one metric per process invocation (src/main.cpp:271-286,
// each computeMetric re-creating its buffers, e.g. src/gpu/fsim/fsim.cpp:279-282); this is the
// batch form of that loop.  Scores are laid out metric by metric in the order SSIM (1 per pair),
// FSIM (2 per pair: FSIM, FSIMc), FLIP (1), M-SVD (1), for the metrics in the mask.
#include <algorithm>
#include <cstring>
#include <vector>

#include "iqm_internal.cuh"

namespace {

constexpr int kMetrics[4] = {IQM_METRIC_SSIM, IQM_METRIC_FSIM, IQM_METRIC_FLIP, IQM_METRIC_MSVD};
constexpr int kScores[4] = {1, 2, 1, 1};

void swap_buf(iqm::DevBuf &a, iqm::DevBuf &b) {
    std::swap(a.ptr, b.ptr);
    std::swap(a.cap, b.cap);
}

// While alive, the context's descriptor and scratch buffers are the caller's (a plan's own, so a
// captured graph keeps pointing at memory nothing else reuses) and FSIM uses the given shapes.
struct BorrowBuffers {
    iqm_ctx *ctx;
    iqm::DevBuf &desc, &scratch;
    iqm::FsimTune saved;
    BorrowBuffers(iqm_ctx *c, iqm::DevBuf &d, iqm::DevBuf &s, const iqm::FsimTune &t)
        : ctx(c), desc(d), scratch(s), saved(c->fsim_tune) {
        swap_buf(ctx->desc, desc);
        swap_buf(ctx->scratch, scratch);
        ctx->fsim_tune = t;
    }
    ~BorrowBuffers() {
        swap_buf(ctx->desc, desc);
        swap_buf(ctx->scratch, scratch);
        ctx->fsim_tune = saved;
    }
};

struct BatchArgs {
    int mask = 0;
    iqm_ssim_params ssim{};
    iqm_flip_params flip{};
    iqm_precision precision = IQM_FP32;
    int energy_mode = 0;
};

int scores_per_pair(int mask) {
    int k = 0;
    for (int m = 0; m < 4; m++)
        if (mask & kMetrics[m]) k += kScores[m];
    return k;
}

void check_batch_args(int mask, const iqm_pair *pairs, int n) {
    IQM_REQUIRE(mask != 0 && (mask & ~(IQM_METRIC_SSIM | IQM_METRIC_FSIM | IQM_METRIC_FLIP | IQM_METRIC_MSVD)) == 0,
                "metric_mask must be a non-empty combination of IQM_METRIC_* flags");
    IQM_REQUIRE(pairs != nullptr && n >= 1, "pairs is NULL or n < 1");
}

// Enqueues metric m (index into kMetrics) for device pairs; scores at `d_scores`.
void enqueue_metric(iqm_ctx *ctx, int m, const BatchArgs &a, const iqm_pair *pairs, int n, double *d_scores) {
    switch (m) {
        case 0: iqm::enqueue_ssim_dev(ctx, pairs, n, &a.ssim, d_scores); break;
        case 1: iqm::enqueue_fsim_dev(ctx, pairs, n, a.precision, a.energy_mode, d_scores); break;
        case 2: iqm::enqueue_flip_dev(ctx, pairs, n, &a.flip, d_scores); break;
        default: iqm::enqueue_msvd_dev(ctx, pairs, n, d_scores); break;
    }
}

BatchArgs resolve_args(int mask, const iqm_ssim_params *sp, const iqm_flip_params *fp, iqm_precision precision,
                       int energy_mode) {
    BatchArgs a;
    a.mask = mask;
    iqm_ssim_default_params(&a.ssim);
    iqm_flip_default_params(&a.flip);
    if (sp) a.ssim = *sp;
    if (fp) a.flip = *fp;
    a.precision = precision;
    a.energy_mode = energy_mode;
    return a;
}

}  // namespace

struct iqm_batch_plan {
    iqm_ctx *ctx = nullptr;
    BatchArgs args;
    std::vector<iqm_pair> pairs;
    double *d_scores = nullptr;
    iqm::DevBuf desc[4], scratch[4];
    iqm::FsimTune tune;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int launches = 0;
    std::string info;

    // Enqueues every metric of the mask (or only metric index `only`) with the plan's buffers;
    // returns the kernel launches.
    int enqueue(const iqm::FsimTune &t, int only = -1) {
        int total = 0;
        double *out = d_scores;
        const int n = int(pairs.size());
        for (int m = 0; m < 4; m++) {
            if (!(args.mask & kMetrics[m])) continue;
            if (only < 0 || only == m) {
                BorrowBuffers b(ctx, desc[m], scratch[m], t);
                ctx->launches = 0;
                enqueue_metric(ctx, m, args, pairs.data(), n, out);
                total += ctx->launches;
            }
            out += size_t(kScores[m]) * n;
        }
        return total;
    }

    // Milliseconds of one FSIM enqueue with shapes t (after one untimed run that sizes buffers).
    float time_fsim(const iqm::FsimTune &t, cudaEvent_t e0, cudaEvent_t e1) {
        enqueue(t, 1);
        IQM_CHECK_CUDA(cudaEventRecord(e0, ctx->stream));
        enqueue(t, 1);
        enqueue(t, 1);
        IQM_CHECK_CUDA(cudaEventRecord(e1, ctx->stream));
        IQM_CHECK_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        IQM_CHECK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return ms / 2.f;
    }

    // Coordinate search over the FSIM shapes: L2 budget of an inverse-pass chunk, warps per CTA of
    // the inverse column pass, rows per CTA of the inverse row pass.  A candidate must be 2% faster
    // to replace the current choice.
    void autotune_fsim() {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        IQM_CHECK_CUDA(cudaEventCreate(&e0));
        IQM_CHECK_CUDA(cudaEventCreate(&e1));
        try {
            iqm::FsimTune best{};
            float best_ms = time_fsim(best, e0, e1);
            auto consider = [&](iqm::FsimTune t) {
                const float ms = time_fsim(t, e0, e1);
                if (ms < best_ms * 0.98f) {
                    best_ms = ms;
                    best = t;
                }
            };
            for (int mb : {40, 160}) {
                iqm::FsimTune t = best;
                t.chunk_mb = mb;
                consider(t);
            }
            const iqm::FsimTune base = best;
            for (int lw : {2, 1}) {
                iqm::FsimTune t = base;
                t.icols_lw = lw;
                consider(t);
            }
            {
                iqm::FsimTune t = best;
                t.rows_per_cta = 1;
                consider(t);
            }
            tune = best;
            char line[160];
            std::snprintf(line, sizeof(line), "fsim: chunk_mb=%d icols_lw=%d rows_per_cta=%d (%.3f ms per batch)",
                          tune.chunk_mb ? tune.chunk_mb : 80, tune.icols_lw, tune.rows_per_cta, double(best_ms));
            info += line;
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }

    void capture() {
        IQM_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
        IQM_CHECK_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        ctx->capturing = true;
        try {
            launches = enqueue(tune);
        } catch (...) {
            ctx->capturing = false;
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(ctx->stream, &g);
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            throw;
        }
        ctx->capturing = false;
        IQM_CHECK_CUDA(cudaStreamEndCapture(ctx->stream, &graph));
        IQM_CHECK_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    }

    void release() {
        if (ctx) cudaStreamSynchronize(ctx->stream);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        for (int m = 0; m < 4; m++) {
            desc[m].release();
            scratch[m].release();
        }
    }
};

#define IQM_API extern "C" __attribute__((visibility("default")))

IQM_API int iqm_batch(iqm_ctx *ctx, int metric_mask, const iqm_pair *pairs, int n, const iqm_ssim_params *ssim,
                      const iqm_flip_params *flip, iqm_precision precision, int energy_mode, double *scores) {
    return iqm::guarded(ctx, [&] {
        check_batch_args(metric_mask, pairs, n);
        IQM_REQUIRE(scores != nullptr, "scores is NULL");
        const BatchArgs a = resolve_args(metric_mask, ssim, flip, precision, energy_mode);
        const int k = scores_per_pair(metric_mask);
        auto *d_scores = static_cast<double *>(ctx->scores.get(sizeof(double) * size_t(k) * n, ctx->stream));
        // scores metric by metric (n per metric, 2n for FSIM); each chunk of pairs fills its slice
        iqm::upload_pipelined(ctx, pairs, n, [&](const iqm_pair *dev, int first, int count) {
            double *out = d_scores;
            for (int m = 0; m < 4; m++) {
                if (!(metric_mask & kMetrics[m])) continue;
                enqueue_metric(ctx, m, a, dev, count, out + size_t(kScores[m]) * first);
                out += size_t(kScores[m]) * n;
            }
        });
        IQM_CHECK_CUDA(cudaMemcpyAsync(scores, d_scores, sizeof(double) * size_t(k) * n, cudaMemcpyDeviceToHost,
                                       ctx->stream));
        IQM_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

IQM_API int iqm_batch_plan_create(iqm_ctx *ctx, int metric_mask, const iqm_pair *dev_pairs, int n,
                                  const iqm_ssim_params *ssim, const iqm_flip_params *flip, iqm_precision precision,
                                  int energy_mode, int autotune, double *d_scores, iqm_batch_plan **out) {
    if (out) *out = nullptr;
    iqm_batch_plan *plan = nullptr;
    const int rc = iqm::guarded(ctx, [&] {
        check_batch_args(metric_mask, dev_pairs, n);
        IQM_REQUIRE(out != nullptr, "out is NULL");
        IQM_REQUIRE(d_scores != nullptr, "d_scores is NULL");
        IQM_REQUIRE(!ctx->capturing, "a batch plan is already being built on this context");
        plan = new iqm_batch_plan();
        plan->ctx = ctx;
        plan->args = resolve_args(metric_mask, ssim, flip, precision, energy_mode);
        plan->pairs.assign(dev_pairs, dev_pairs + n);
        plan->d_scores = d_scores;
        // validates every metric's arguments, sizes the plan's buffers and builds per-size tables
        plan->enqueue(plan->tune);
        if (autotune && (metric_mask & IQM_METRIC_FSIM)) {
            plan->autotune_fsim();
            plan->enqueue(plan->tune);  // buffers sized for the chosen shapes
        } else {
            plan->info += "fsim: default shapes";
        }
        plan->capture();
        ctx->launches = plan->launches;
    });
    if (rc != IQM_OK) {
        if (plan) {
            plan->release();
            delete plan;
        }
        return rc;
    }
    *out = plan;
    return IQM_OK;
}

IQM_API int iqm_batch_plan_run(iqm_batch_plan *plan) {
    if (!plan) return IQM_EINVAL;
    iqm_ctx *ctx = plan->ctx;
    return iqm::guarded(ctx, [&] {
        IQM_CHECK_CUDA(cudaGraphLaunch(plan->exec, ctx->stream));
        ctx->launches = plan->launches;
    });
}

IQM_API int iqm_batch_plan_info(const iqm_batch_plan *plan, char *buf, size_t cap, int *launches) {
    if (!plan || !buf || cap == 0) return IQM_EINVAL;
    std::snprintf(buf, cap, "%s", plan->info.c_str());
    if (launches) *launches = plan->launches;
    return plan->info.size() < cap ? IQM_OK : IQM_EINVAL;
}

IQM_API int iqm_batch_plan_destroy(iqm_batch_plan *plan) {
    if (!plan) return IQM_EINVAL;
    if (plan->ctx) cudaSetDevice(plan->ctx->device);
    plan->release();
    delete plan;
    return IQM_OK;
}
