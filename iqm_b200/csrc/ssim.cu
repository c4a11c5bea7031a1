// SSIM / MSSIM on sm_100a: one fused kernel per batch of pairs.
//
// Reference path (cadik/IQM): three full-image Vulkan dispatches and a host pass --
//   luma pack        shaders/ssim/ssim_lumapack.glsl:19-35   (0.299 R + 0.581 G + 0.114 B, unorm)
//   Gaussian means   shaders/ssim/ssim_gaussinput.glsl:22-57 (11x11 window, truncated at the image
//                    border and renormalised by the in-image weight sum)
//   variances + map  shaders/ssim/ssim.glsl:25-79           (same window, two-pass form)
//   MSSIM            src/gpu/ssim/ssim.cpp:386-401           (x, y in [r, dim - r], host double sum)
//
// This kernel computes the same quantities in one pass over the RGBA8 inputs:
//   * the 2-D window is separable, w(dx,dy) = g(dx) g(dy), and so is its truncation: the in-image
//     weight sum of pixel (x,y) is wx(x) * wy(y);
//   * with u = a + b and v = a - b the five SSIM moments reduce to four (mean and second moment
//     of u and v): mu_a mu_b = (mu_u^2 - mu_v^2)/4, mu_a^2 + mu_b^2 = (mu_u^2 + mu_v^2)/2,
//     cov_ab = (var_u - var_v)/4, var_a + var_b = (var_u + var_v)/2;
//   * the second moments are taken about a per-tile constant (the u, v of the tile's centre
//     pixel), var = E[(x-c)^2] - E[x-c]^2, which keeps FP32 cancellation ~1e-7 on MSSIM;
//   * each CTA owns a 128-column strip of ~120 output rows and streams down it: raw RGBA8 rows
//     (plus a 5-pixel halo) are prefetched PF rows ahead with cp.async into a small shared ring,
//     converted once to shifted (u, v), filtered horizontally from shared memory and pushed into a
//     register ring of 2R+1 rows that carries the vertical taps (one barrier per row, ~11 KB of
//     shared memory per CTA, so many CTAs overlap their loads with arithmetic);
//   * (u, v) pairs are processed with packed FP32x2 instructions (__ffma2_rn and friends);
//   * MSSIM partials go to per-tile FP64 slots; the last CTA of a pair sums them in a fixed order
//     (deterministic, no second launch).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "iqm_internal.cuh"

namespace {

constexpr int TW = 128;             // output columns per CTA (one vertical strip)
constexpr int NT = TW;              // threads per CTA, one output column each
constexpr int SMEM_COLS = TW + 16;  // staged columns x0-8 .. x0+TW+7 (16-byte aligned start)
constexpr int NRAW = 8;             // raw RGBA row ring
constexpr int PF = 6;               // rows prefetched ahead (< NRAW)

template <int R>
struct Geom {
    static constexpr int K = 2 * R + 1;
    // strip height: S + 2R is a multiple of K so the register ring indexes statically
    static constexpr int S = K * ((120 + 2 * R + K - 1) / K) - 2 * R;
    static constexpr int ROWS = S + 2 * R;
};

struct Smem {
    uint32_t raw[NRAW][2][SMEM_COLS];  // RGBA8 rows of both images, as loaded
    float2 uv[2][SMEM_COLS];           // shifted (u, v) of the row being filtered
};

struct SsimPairDev {
    const uint8_t *a;
    const uint8_t *b;
    float *map;        // nullable
    long long pitch;   // bytes between rows (both images)
    int w, h;
    int tiles_x;
    int tile_base;     // first global tile index of this pair
    int ntiles;
    int vec_ok;        // 16-byte loads allowed
    int unit_base;     // tensor-core kernel: first global work unit (column segment of tiles)
};

struct SsimArgs {
    const SsimPairDev *pairs;
    int npairs;
    double *partials;    // one per tile
    unsigned *counters;  // one per pair, zero on entry
    double *scores;      // one per pair
    float g[15];         // 1-D Gaussian taps g(-R..R)
    float c1, c2;
};

// shaders/ssim/ssim_lumapack.glsl:19-21 (G weight 0.581 as in the reference) on unorm bytes
__device__ __forceinline__ float luma_u8(uint32_t px) {
    float r = float(px & 0xffu) * (1.0f / 255.0f);
    float g = float((px >> 8) & 0xffu) * (1.0f / 255.0f);
    float b = float((px >> 16) & 0xffu) * (1.0f / 255.0f);
    return 0.299f * r + 0.581f * g + 0.114f * b;
}

__device__ __forceinline__ int find_pair(const SsimPairDev *pairs, int n, int tile) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (pairs[mid].tile_base <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src, int src_bytes) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
// "memory" clobbers: the compiler must not move shared-memory accesses across the copies or waits
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Issue the copies of image row y (both images, staged columns) into raw ring slot `slot`.
// Columns or rows outside the image are not fetched: the conversion step zeroes them.
__device__ __forceinline__ void issue_row(Smem &sm, const SsimPairDev &P, int x0, int y, int slot) {
    if (y < 0 || y >= P.h) return;
    const int xs = x0 - 8;
    if (P.vec_ok) {
        constexpr int CH = SMEM_COLS / 4;  // 16-byte chunks per image row
        for (int c = threadIdx.x; c < 2 * CH; c += NT) {
            const int img = c / CH, q = c - img * CH;
            const int x = xs + 4 * q;
            if (x < 0 || x >= P.w) continue;
            const int valid = min(4, P.w - x);
            const uint8_t *src = (img ? P.b : P.a) + (long long)y * P.pitch + 4LL * x;
            cp_async16(&sm.raw[slot][img][4 * q], src, 4 * valid);
        }
    } else {
        for (int c = threadIdx.x; c < 2 * SMEM_COLS; c += NT) {
            const int img = c / SMEM_COLS, q = c - img * SMEM_COLS;
            const int x = xs + q;
            if (x < 0 || x >= P.w) continue;
            const uint8_t *src = (img ? P.b : P.a) + (long long)y * P.pitch + 4LL * x;
            cp_async4(&sm.raw[slot][img][q], src);
        }
    }
}

// Raw RGBA row -> shifted (u, v) row; positions outside the image become (0, 0), which removes
// them from every window sum (the reference skips out-of-image taps).
__device__ __forceinline__ void convert_row(Smem &sm, const SsimPairDev &P, int x0, int y, int slot,
                                            float2 *dst, float cu, float cv) {
    const bool row_ok = y >= 0 && y < P.h;
    for (int q = threadIdx.x; q < SMEM_COLS; q += NT) {
        const int x = x0 - 8 + q;
        float2 o = make_float2(0.f, 0.f);
        if (row_ok && x >= 0 && x < P.w) {
            const float la = luma_u8(sm.raw[slot][0][q]), lb = luma_u8(sm.raw[slot][1][q]);
            o = make_float2((la + lb) - cu, (la - lb) - cv);
        }
        dst[q] = o;
    }
}

// Deterministic pooling, shared by the SSIM kernels: the CTA's partial (FP64, fixed order) goes to
// its tile slot; the last CTA of the pair to finish sums the pair's slots in a fixed order and
// writes the mean (`count` pooled pixels).  `red` holds NTH/32 doubles of shared memory.
template <int NTH>
__device__ __forceinline__ void pool_tiles(float acc, double *red, int *is_last, double *partials,
                                           unsigned *counters, double *scores, int pi, const SsimPairDev &P,
                                           int gt, double count) {
    const int tid = threadIdx.x;
    double d = double(acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_down_sync(0xffffffffu, d, o);
    if ((tid & 31) == 0) red[tid >> 5] = d;
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < NTH / 32; i++) s += red[i];
        partials[gt] = s;
        __threadfence();
        const unsigned prev = atomicAdd(&counters[pi], 1u);
        *is_last = (prev == unsigned(P.ntiles - 1));
    }
    __syncthreads();
    if (!*is_last) return;
    __threadfence();
    double s = 0.0;
    for (int i = tid; i < P.ntiles; i += NTH) s += __ldcg(&partials[P.tile_base + i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __syncthreads();
    if ((tid & 31) == 0) red[tid >> 5] = s;
    __syncthreads();
    if (tid == 0) {
        double tot = 0.0;
#pragma unroll
        for (int i = 0; i < NTH / 32; i++) tot += red[i];
        scores[pi] = tot / count;
        counters[pi] = 0u;  // ready for the next launch
    }
}

template <int R>
// 8 CTAs of 128 threads per SM (at most 64 registers a thread): the row pipeline is latency-bound,
// so resident warps matter more than registers per thread.
__global__ void __launch_bounds__(NT, 8) ssim_kernel(SsimArgs args) {
    using G = Geom<R>;
    constexpr int K = G::K, S = G::S, ROWS = G::ROWS;
    __shared__ __align__(16) Smem sm;
    __shared__ double red[NT / 32];
    __shared__ int is_last;

    const int gt = blockIdx.x;
    const int pi = find_pair(args.pairs, args.npairs, gt);
    const SsimPairDev P = args.pairs[pi];
    const int local = gt - P.tile_base;
    const int x0 = (local % P.tiles_x) * TW;
    const int y0 = (local / P.tiles_x) * S;
    const int W = P.w, H = P.h;
    const int tid = threadIdx.x;

    // prefetch the first PF rows (tile row r = image row y0 - R + r)
#pragma unroll
    for (int r = 0; r < PF; r++) {
        issue_row(sm, P, x0, y0 - R + r, r % NRAW);
        cp_async_commit();
    }

    // per-tile shift constants: u, v of the tile's centre pixel (keeps FP32 cancellation small)
    float cu, cv;
    {
        const int cx = min(x0 + TW / 2, W - 1), cy = min(y0 + S / 2, H - 1);
        const uint32_t pa = __ldg(reinterpret_cast<const uint32_t *>(P.a + (long long)cy * P.pitch) + cx);
        const uint32_t pb = __ldg(reinterpret_cast<const uint32_t *>(P.b + (long long)cy * P.pitch) + cx);
        const float la = luma_u8(pa), lb = luma_u8(pb);
        cu = la + lb;
        cv = la - lb;
    }

    cp_async_wait<PF - 1>();
    __syncthreads();
    convert_row(sm, P, x0, y0 - R, 0, sm.uv[0], cu, cv);
    issue_row(sm, P, x0, y0 - R + PF, PF % NRAW);
    cp_async_commit();

    const int col0 = tid;                // this thread's tile column
    const int start = col0 + 8 - R;      // staged index of its leftmost horizontal tap
    float gsum = 0.f;
#pragma unroll
    for (int k = 0; k < K; k++) gsum += args.g[k];
    constexpr int CPT = 1;
    float rwx[CPT];
#pragma unroll
    for (int c = 0; c < CPT; c++) {
        const int x = x0 + col0 + c;
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int xx = x + k - R;
            s += (xx >= 0 && xx < W) ? args.g[k] : 0.f;
        }
        rwx[c] = 1.0f / s;
    }

    float2 ring_m[CPT][K];  // (sum g u, sum g v) of the last K rows, per column
    float2 ring_s[CPT][K];  // (sum g u^2, sum g v^2)
    float acc = 0.f;      // pooled SSIM of this thread
    bool col_in[CPT];
#pragma unroll
    for (int c = 0; c < CPT; c++) col_in[c] = x0 + col0 + c < W;

    for (int jb = 0; jb < ROWS; jb += K) {
#pragma unroll
        for (int t = 0; t < K; t++) {
            const int j = jb + t;
            // make row j+1 available: wait for its copies, convert it, prefetch row j+1+PF
            cp_async_wait<PF - 1>();
            __syncthreads();
            if (j + 1 < ROWS) convert_row(sm, P, x0, y0 - R + j + 1, (j + 1) % NRAW, sm.uv[(j + 1) & 1], cu, cv);
            if (j + 1 + PF < ROWS) issue_row(sm, P, x0, y0 - R + j + 1 + PF, (j + 1 + PF) % NRAW);
            cp_async_commit();

            // horizontal taps of row j
            float2 v[K];
#pragma unroll
            for (int q = 0; q < K; q++) v[q] = sm.uv[j & 1][start + q];
#pragma unroll
            for (int c = 0; c < CPT; c++) {
                float2 hm = make_float2(0.f, 0.f), hs = make_float2(0.f, 0.f);
#pragma unroll
                for (int k = 0; k < K; k++) {
                    const float2 sv = v[c + k];
                    const float2 gs = __fmul2_rn(make_float2(args.g[k], args.g[k]), sv);
                    hm = __fadd2_rn(hm, gs);
                    hs = __ffma2_rn(gs, sv, hs);
                }
                ring_m[c][t] = hm;
                ring_s[c][t] = hs;
            }
            if (j >= 2 * R) {
                // vertical taps: output row i = j - 2R uses tile rows i .. i + 2R
                const int y = y0 + j - 2 * R;
                if (y < H) {
                    float wy = gsum;
                    if (y < R || y >= H - R) {
                        wy = 0.f;
#pragma unroll
                        for (int k = 0; k < K; k++) {
                            const int yy = y + k - R;
                            wy += (yy >= 0 && yy < H) ? args.g[k] : 0.f;
                        }
                    }
                    const float rwy = 1.0f / wy;
                    const bool pool_y = y >= R && y <= H - R;
#pragma unroll
                    for (int c = 0; c < CPT; c++) {
                        float2 mm = make_float2(0.f, 0.f), ms = make_float2(0.f, 0.f);
#pragma unroll
                        for (int k = 0; k < K; k++) {
                            const int slot = (t + 1 + k) % K;
                            const float2 gk = make_float2(args.g[k], args.g[k]);
                            mm = __ffma2_rn(gk, ring_m[c][slot], mm);
                            ms = __ffma2_rn(gk, ring_s[c][slot], ms);
                        }
                        if (col_in[c]) {
                            const int x = x0 + col0 + c;
                            const float inv = rwx[c] * rwy;
                            const float su = mm.x * inv, sv = mm.y * inv;  // shifted means
                            const float varu = fmaf(ms.x, inv, -su * su);
                            const float varv = fmaf(ms.y, inv, -sv * sv);
                            const float mu = su + cu, mv = sv + cv;
                            const float mu2 = mu * mu, mv2 = mv * mv;
                            const float num = (0.5f * (mu2 - mv2) + args.c1) * (0.5f * (varu - varv) + args.c2);
                            const float den = (0.5f * (mu2 + mv2) + args.c1) * (0.5f * (varu + varv) + args.c2);
                            const float ssim = num * iqm::rcp_approx(den);  // den >= c1 c2 > 0
                            if (P.map) P.map[(long long)y * W + x] = ssim;
                            if (pool_y && x >= R && x <= W - R) acc += ssim;
                        }
                    }
                }
            }
        }
    }
    cp_async_wait<0>();
    pool_tiles<NT>(acc, red, &is_last, args.partials, args.counters, args.scores, pi, P, gt,
                   double(W - 2 * R + 1) * double(H - 2 * R + 1));
}

}  // namespace

#include "ssim_mma.cuh"

namespace {

template <int R>
void launch_ssim(const SsimArgs &a, int total_tiles, cudaStream_t s) {
    ssim_kernel<R><<<total_tiles, NT, 0, s>>>(a);
}

int strip_rows(int R) {
    switch (R) {
        case 1: return Geom<1>::S;
        case 2: return Geom<2>::S;
        case 3: return Geom<3>::S;
        case 4: return Geom<4>::S;
        case 5: return Geom<5>::S;
        case 6: return Geom<6>::S;
        default: return Geom<7>::S;
    }
}

void check_params(const iqm_ssim_params &p) {
    int R = (p.kernel_size - 1) / 2;
    IQM_REQUIRE(R >= 1 && R <= 7, "kernel_size must give a radius (kernel_size-1)/2 in [1, 7]");
    IQM_REQUIRE(p.sigma > 0.f && std::isfinite(p.sigma), "sigma must be positive");
    IQM_REQUIRE(std::isfinite(p.k1) && std::isfinite(p.k2), "k1/k2 must be finite");
    IQM_REQUIRE(p.precision == IQM_FP32 || p.precision == IQM_MIXED || p.precision == IQM_MIXED_FAST,
                "unknown precision " + std::to_string(p.precision));
}

// The tensor-core kernel (one 64x32 tile per CTA) for IQM_MIXED (split products) and
// IQM_MIXED_FAST (single products).
// Persistent launch: as many CTAs as fit on the device at once (at most one per work unit).
template <int SPLIT>
void launch_ssim_mma(const SsimMmaArgs &a, int total_units, int device, cudaStream_t s) {
    const size_t smem = SsimMmaGeom<SPLIT>::smem_bytes;
    IQM_CHECK_CUDA(cudaFuncSetAttribute(ssim_mma_kernel<SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    int sms = 0, per_sm = 0;
    IQM_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    IQM_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ssim_mma_kernel<SPLIT>, MT_THREADS, smem));
    const int grid = std::max(1, std::min(total_units, sms * std::max(1, per_sm)));
    ssim_mma_kernel<SPLIT><<<grid, MT_THREADS, smem, s>>>(a, total_units);
}

// Enqueue SSIM for device-resident pairs; `maps[i]` (device, nullable) receive the SSIM maps.
void ssim_enqueue(iqm_ctx *ctx, const std::vector<iqm_pair> &pairs, const iqm_ssim_params &p,
                  const std::vector<float *> &maps, double *d_scores) {
    const int n = int(pairs.size());
    const int R = (p.kernel_size - 1) / 2;
    const bool mma = p.precision != IQM_FP32;
    const int tw = mma ? MT_W : TW, th = mma ? MT_H : strip_rows(R);
    std::vector<SsimPairDev> hd(n);
    int total = 0, units = 0;
    const int segt = MT_SEG_SPLIT;  // tensor-core kernel: tiles per column segment (work unit)
    for (int i = 0; i < n; i++) {
        const iqm_pair &q = pairs[i];
        SsimPairDev &d = hd[i];
        d.a = q.input;
        d.b = q.ref;
        d.map = maps.empty() ? nullptr : maps[i];
        d.pitch = (long long)q.row_bytes;
        d.w = q.w;
        d.h = q.h;
        d.tiles_x = int(iqm::ceil_div(q.w, tw));
        d.ntiles = d.tiles_x * int(iqm::ceil_div(q.h, th));
        d.tile_base = total;
        d.vec_ok = ((reinterpret_cast<uintptr_t>(q.input) | reinterpret_cast<uintptr_t>(q.ref) |
                     uintptr_t(q.row_bytes)) & 15u) == 0;
        d.unit_base = units;
        total += d.ntiles;
        units += d.tiles_x * int(iqm::ceil_div(d.ntiles / d.tiles_x, segt));
    }
    auto *d_desc = static_cast<SsimPairDev *>(
        iqm::upload_bytes(ctx, ctx->desc, hd.data(), sizeof(SsimPairDev) * n));
    const size_t part_bytes = (sizeof(double) * total + 255) & ~size_t(255);
    const size_t cnt_bytes = (sizeof(unsigned) * n + 255) & ~size_t(255);
    auto *scr = static_cast<uint8_t *>(ctx->scratch.get(part_bytes + cnt_bytes, ctx->stream));
    double g64[15] = {}, gsum = 0.0;
    for (int k = -R; k <= R; k++) gsum += (g64[k + R] = std::exp(-double(k * k) / (2.0 * double(p.sigma) * p.sigma)));
    auto *counters = reinterpret_cast<unsigned *>(scr + part_bytes);
    IQM_CHECK_CUDA(cudaMemsetAsync(counters, 0, sizeof(unsigned) * n, ctx->stream));
    iqm::timing_mark(ctx, nullptr);
    if (mma) {
        SsimMmaArgs a{};
        a.pairs = d_desc;
        a.npairs = n;
        a.R = R;
        a.partials = reinterpret_cast<double *>(scr);
        a.counters = counters;
        a.scores = d_scores;
        for (int k = 0; k < 15; k++) a.gn[k] = float(g64[k] / gsum);
        a.c1 = p.k1 * p.k1;
        a.c2 = p.k2 * p.k2;
        if (p.precision == IQM_MIXED) launch_ssim_mma<3>(a, units, ctx->device, ctx->stream);
        else launch_ssim_mma<1>(a, units, ctx->device, ctx->stream);
        iqm::check_launch(ctx, "ssim_mma_kernel");
        return;
    }
    SsimArgs a{};
    a.pairs = d_desc;
    a.npairs = n;
    a.partials = reinterpret_cast<double *>(scr);
    a.counters = counters;
    a.scores = d_scores;
    for (int k = 0; k < 15; k++) a.g[k] = float(g64[k]);
    a.c1 = p.k1 * p.k1;
    a.c2 = p.k2 * p.k2;
    switch (R) {
        case 1: launch_ssim<1>(a, total, ctx->stream); break;
        case 2: launch_ssim<2>(a, total, ctx->stream); break;
        case 3: launch_ssim<3>(a, total, ctx->stream); break;
        case 4: launch_ssim<4>(a, total, ctx->stream); break;
        case 5: launch_ssim<5>(a, total, ctx->stream); break;
        case 6: launch_ssim<6>(a, total, ctx->stream); break;
        default: launch_ssim<7>(a, total, ctx->stream); break;
    }
    iqm::check_launch(ctx, "ssim_kernel");
}

iqm_ssim_params resolve(const iqm_ssim_params *p) {
    iqm_ssim_params d;
    iqm_ssim_default_params(&d);
    return p ? *p : d;
}

}  // namespace

extern "C" __attribute__((visibility("default"))) void iqm_ssim_default_params(iqm_ssim_params *p) {
    if (!p) return;
    // src/gpu/ssim/ssim.h:31-34
    p->kernel_size = 11;
    p->k1 = 0.01f;
    p->k2 = 0.03f;
    p->sigma = 1.5f;
    p->precision = IQM_FP32;
}

void iqm::enqueue_ssim_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n, const iqm_ssim_params *params,
                           double *d_scores) {
    const iqm_ssim_params p = resolve(params);
    check_params(p);
    const int R = (p.kernel_size - 1) / 2;
    iqm::check_pairs(pairs, n, R, R);
    iqm::check_dev_alignment(pairs, n);
    IQM_REQUIRE(d_scores != nullptr, "d_scores is NULL");
    ssim_enqueue(ctx, std::vector<iqm_pair>(pairs, pairs + n), p, {}, d_scores);
}

extern "C" __attribute__((visibility("default"))) int iqm_ssim_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n, const iqm_ssim_params *params,
                            double *d_scores) {
    return iqm::guarded(ctx, [&] { iqm::enqueue_ssim_dev(ctx, pairs, n, params, d_scores); });
}

extern "C" __attribute__((visibility("default"))) int iqm_ssim_batch(iqm_ctx *ctx, const iqm_pair *pairs, int n, const iqm_ssim_params *params,
                              double *scores) {
    return iqm::guarded(ctx, [&] {
        const iqm_ssim_params p = resolve(params);
        check_params(p);
        const int R = (p.kernel_size - 1) / 2;
        iqm::check_pairs(pairs, n, R, R);
        IQM_REQUIRE(scores != nullptr, "scores is NULL");
        auto *d_scores = static_cast<double *>(ctx->scores.get(sizeof(double) * n, ctx->stream));
        iqm::upload_pipelined(ctx, pairs, n, [&](const iqm_pair *dev, int first, int count) {
            ssim_enqueue(ctx, std::vector<iqm_pair>(dev, dev + count), p, {}, d_scores + first);
        });
        IQM_CHECK_CUDA(cudaMemcpyAsync(scores, d_scores, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
        IQM_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

extern "C" __attribute__((visibility("default"))) int iqm_ssim(iqm_ctx *ctx, const uint8_t *rgba_in, const uint8_t *rgba_ref, int w, int h,
                        size_t row_bytes, const iqm_ssim_params *params, float *map_out, double *mssim) {
    return iqm::guarded(ctx, [&] {
        const iqm_ssim_params p = resolve(params);
        check_params(p);
        IQM_REQUIRE(mssim != nullptr, "mssim is NULL");
        const int R = (p.kernel_size - 1) / 2;
        iqm_pair hp{rgba_in, rgba_ref, w, h, row_bytes};
        iqm::check_pairs(&hp, 1, R, R);
        auto dev = iqm::upload_pairs(ctx, &hp, 1);
        auto *d_score = static_cast<double *>(ctx->scores.get(sizeof(double), ctx->stream));
        std::vector<float *> maps;
        float *d_map = nullptr;
        if (map_out) {
            d_map = static_cast<float *>(ctx->maps.get(sizeof(float) * size_t(w) * h, ctx->stream));
            maps.push_back(d_map);
        }
        ssim_enqueue(ctx, dev, p, maps, d_score);
        IQM_CHECK_CUDA(cudaMemcpyAsync(mssim, d_score, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        if (map_out)
            IQM_CHECK_CUDA(cudaMemcpyAsync(map_out, d_map, sizeof(float) * size_t(w) * h,
                                           cudaMemcpyDeviceToHost, ctx->stream));
        IQM_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

// ---------------------------------------------------------------------------------------------
// Allocation-free SSIM.  Some callers cannot let a library allocate device memory: a host
// application that reserves the whole GPU for its own allocator, or a plugin whose host accounts
// for every byte it hands out.  iqm_ssim_noalloc serves them: the caller passes device inputs and
// outputs, and the kernel's scratch (pair descriptor, completion counter, per-tile partial sums)
// lives in the fixed array below, which every GPU that loads this library holds until exit.
namespace {

struct NoallocScratch {
    SsimPairDev desc;                                 // the pair of the current call
    unsigned counter;                                 // CTAs finished; must be 0 at launch
    double partials[IQM_SSIM_NOALLOC_MAX_TILES];      // one per tile
};

static __device__ __align__(256) unsigned char g_ssim_noalloc_scratch[sizeof(NoallocScratch)];

// Host-side copies of the array's device address, one per device, filled on the first call made
// with that device current.  In host code the symbol itself is only a stand-in, not an address.
constexpr int NOALLOC_MAX_DEVICES = 64;
void *g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};
std::mutex g_noalloc_mu;

// Writes the descriptor and clears the counter (the array keeps the previous call's contents).
__global__ void ssim_noalloc_setup_kernel(NoallocScratch *s, SsimPairDev d) {
    s->desc = d;
    s->counter = 0u;
}

// Launches ssim_kernel<R> and returns that launch's own status.  cudaLaunchKernel reports errors of
// this launch only, so an error left pending by the caller's earlier work is neither returned nor
// cleared here; a failed launch's own error is cleared before returning.
template <int R>
cudaError_t launch_ssim_checked(SsimArgs &a, int total_tiles, cudaStream_t st) {
    void *args[] = {&a};
    const cudaError_t e = cudaLaunchKernel((const void *)ssim_kernel<R>, dim3(total_tiles), dim3(NT), args, 0, st);
    if (e != cudaSuccess) cudaGetLastError();
    return e;
}

}  // namespace

extern "C" __attribute__((visibility("default"))) int iqm_ssim_noalloc(
    const uint8_t *d_in, const uint8_t *d_ref, int w, int h, size_t row_bytes, const iqm_ssim_params *params,
    float *d_map, double *d_mssim, void *cuda_stream) {
    if (!d_in || !d_ref || !d_mssim) return IQM_EINVAL;
    // pixels are read as 4-byte words, the score as a double and the map as floats: misaligned
    // pointers would fault on the GPU, so they are refused before any launch
    if (((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_ref) | uintptr_t(row_bytes) |
          reinterpret_cast<uintptr_t>(d_map)) & 3u) != 0 || (reinterpret_cast<uintptr_t>(d_mssim) & 7u) != 0)
        return IQM_EINVAL;
    const iqm_ssim_params p = resolve(params);
    try {
        check_params(p);
    } catch (const iqm::Error &e) {
        return e.code;
    }
    if (p.precision != IQM_FP32) return IQM_EINVAL;  // the fixed scratch is sized for the FP32 tiles
    const int R = (p.kernel_size - 1) / 2;
    if (w < 2 * R || h < 2 * R || w > 65536 || h > 65536 || row_bytes < size_t(w) * 4) return IQM_EINVAL;
    const int tiles_x = int(iqm::ceil_div(w, TW));
    const long tiles = long(tiles_x) * long(iqm::ceil_div(h, strip_rows(R)));
    if (tiles > IQM_SSIM_NOALLOC_MAX_TILES) return IQM_EINVAL;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return IQM_ECUDA;
    void *addr = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            void *a = nullptr;
            if (cudaGetSymbolAddress(&a, g_ssim_noalloc_scratch) != cudaSuccess || !a) {
                cudaGetLastError();  // this lookup's own error
                return IQM_ECUDA;
            }
            g_noalloc_addr[dev] = a;
        }
        addr = g_noalloc_addr[dev];
    }
    auto *s = static_cast<NoallocScratch *>(addr);
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);

    SsimPairDev d{};
    d.a = d_in;
    d.b = d_ref;
    d.map = d_map;
    d.pitch = (long long)row_bytes;
    d.w = w;
    d.h = h;
    d.tiles_x = tiles_x;
    d.tile_base = 0;
    d.ntiles = int(tiles);
    d.vec_ok = ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_ref) | uintptr_t(row_bytes)) &
                15u) == 0;
    {
        void *args[] = {&s, &d};
        const cudaError_t e =
            cudaLaunchKernel((const void *)ssim_noalloc_setup_kernel, dim3(1), dim3(1), args, 0, st);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return IQM_ECUDA;  // the SSIM kernel is not launched without its descriptor
        }
    }

    SsimArgs a{};
    a.pairs = &s->desc;
    a.npairs = 1;
    a.partials = s->partials;
    a.counters = &s->counter;
    a.scores = d_mssim;
    for (int k = 0; k < 15; k++) a.g[k] = 0.f;
    for (int k = -R; k <= R; k++) a.g[k + R] = float(std::exp(-double(k * k) / (2.0 * double(p.sigma) * p.sigma)));
    a.c1 = p.k1 * p.k1;
    a.c2 = p.k2 * p.k2;
    cudaError_t e;
    switch (R) {
        case 1: e = launch_ssim_checked<1>(a, int(tiles), st); break;
        case 2: e = launch_ssim_checked<2>(a, int(tiles), st); break;
        case 3: e = launch_ssim_checked<3>(a, int(tiles), st); break;
        case 4: e = launch_ssim_checked<4>(a, int(tiles), st); break;
        case 5: e = launch_ssim_checked<5>(a, int(tiles), st); break;
        case 6: e = launch_ssim_checked<6>(a, int(tiles), st); break;
        default: e = launch_ssim_checked<7>(a, int(tiles), st); break;
    }
    return e == cudaSuccess ? IQM_OK : IQM_ECUDA;
}
