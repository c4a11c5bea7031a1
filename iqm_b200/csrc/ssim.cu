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
//   * horizontal taps are read from a shared-memory tile (128 output columns + halo, one CTA),
//     vertical taps live in a register ring of 2R+1 rows: each thread slides down its two columns;
//   * MSSIM partials go to per-tile FP64 slots; the last CTA of a pair sums them in a fixed order
//     (deterministic, no second launch).
#include <cmath>
#include <cstring>

#include "iqm_internal.cuh"

namespace {

constexpr int TW = 128;          // output columns per CTA
constexpr int NT = 64;           // threads per CTA; each owns 2 adjacent columns
constexpr int SMEM_COLS = TW + 16;  // tile columns x0-8 .. x0+TW+7 (16-byte aligned start)

template <int R>
struct Geom {
    static constexpr int K = 2 * R + 1;
    // strip height: S + 2R is a multiple of K so the register ring indexes statically
    static constexpr int S = K * ((32 + 2 * R + K - 1) / K) - 2 * R;
    static constexpr int ROWS = S + 2 * R;
    static constexpr size_t SMEM = size_t(ROWS) * SMEM_COLS * sizeof(float2);
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

// shaders/ssim/ssim_lumapack.glsl:155-157 (G weight 0.581 as in the reference) on unorm bytes
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

template <int R>
__global__ void __launch_bounds__(NT, 4) ssim_kernel(SsimArgs args) {
    using G = Geom<R>;
    constexpr int K = G::K, S = G::S, ROWS = G::ROWS;
    extern __shared__ float4 smem_raw[];
    float2 *tile = reinterpret_cast<float2 *>(smem_raw);
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

    // per-tile shift constants: u, v of the tile's centre pixel
    float cu, cv;
    {
        int cx = min(x0 + TW / 2, W - 1), cy = min(y0 + S / 2, H - 1);
        uint32_t pa = __ldg(reinterpret_cast<const uint32_t *>(P.a + (long long)cy * P.pitch) + cx);
        uint32_t pb = __ldg(reinterpret_cast<const uint32_t *>(P.b + (long long)cy * P.pitch) + cx);
        float la = luma_u8(pa), lb = luma_u8(pb);
        cu = la + lb;
        cv = la - lb;
    }

    // ---- stage RGBA8 -> shifted (u, v) for rows y0-R .. y0+S+R-1, columns x0-8 .. x0+TW+7 ----
    {
        constexpr int GROUPS = SMEM_COLS / 4;  // 4-pixel groups per row
        const int xs = x0 - 8;
        for (int idx = tid; idx < ROWS * GROUPS; idx += NT) {
            const int r = idx / GROUPS, gq = idx - r * GROUPS;
            const int y = y0 - R + r, x = xs + 4 * gq;
            float2 out[4];
            if (y < 0 || y >= H || x >= W || x + 3 < 0) {
#pragma unroll
                for (int q = 0; q < 4; q++) out[q] = make_float2(0.f, 0.f);
            } else {
                const uint8_t *ra = P.a + (long long)y * P.pitch;
                const uint8_t *rb = P.b + (long long)y * P.pitch;
                uint32_t pa[4], pb[4];
                if (P.vec_ok && x >= 0 && x + 3 < W) {
                    uint4 va = __ldg(reinterpret_cast<const uint4 *>(ra) + (x >> 2));
                    uint4 vb = __ldg(reinterpret_cast<const uint4 *>(rb) + (x >> 2));
                    pa[0] = va.x; pa[1] = va.y; pa[2] = va.z; pa[3] = va.w;
                    pb[0] = vb.x; pb[1] = vb.y; pb[2] = vb.z; pb[3] = vb.w;
                } else {
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        int xx = x + q;
                        bool ok = xx >= 0 && xx < W;
                        pa[q] = ok ? __ldg(reinterpret_cast<const uint32_t *>(ra) + xx) : 0u;
                        pb[q] = ok ? __ldg(reinterpret_cast<const uint32_t *>(rb) + xx) : 0u;
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    int xx = x + q;
                    if (xx >= 0 && xx < W) {
                        float la = luma_u8(pa[q]), lb = luma_u8(pb[q]);
                        out[q] = make_float2((la + lb) - cu, (la - lb) - cv);
                    } else {
                        out[q] = make_float2(0.f, 0.f);
                    }
                }
            }
            float4 *dst = reinterpret_cast<float4 *>(tile + r * SMEM_COLS + 4 * gq);
            dst[0] = make_float4(out[0].x, out[0].y, out[1].x, out[1].y);
            dst[1] = make_float4(out[2].x, out[2].y, out[3].x, out[3].y);
        }
    }
    __syncthreads();

    // ---- sliding separable window ----
    constexpr int OFF = (8 - R) & 1;        // parity fix so float4 reads stay 16-byte aligned
    constexpr int NV = (2 * R + 4) / 2;     // float4 reads per row (2R+4 float2 values)
    const int col0 = 2 * tid;               // first of this thread's two tile columns
    const int start = col0 + 8 - R - OFF;   // even
    float gsum = 0.f;
#pragma unroll
    for (int k = 0; k < K; k++) gsum += args.g[k];
    float wxv[2];
#pragma unroll
    for (int c = 0; c < 2; c++) {
        const int x = x0 + col0 + c;
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < K; k++) {
            int xx = x + k - R;
            s += (xx >= 0 && xx < W) ? args.g[k] : 0.f;
        }
        wxv[c] = s;
    }

    float ring[2][K][4];
    float acc = 0.f;  // pooled SSIM of this thread (<= 2*S terms)
    const int pool_x_lo = R, pool_x_hi = W - R, pool_y_lo = R, pool_y_hi = H - R;

    for (int jb = 0; jb < ROWS; jb += K) {
#pragma unroll
        for (int t = 0; t < K; t++) {
            const int j = jb + t;  // tile row; image row y0 - R + j
            // horizontal taps
            float2 v[2 * R + 4];
            const float4 *src = reinterpret_cast<const float4 *>(tile + j * SMEM_COLS + start);
#pragma unroll
            for (int q = 0; q < NV; q++) {
                float4 f = src[q];
                v[2 * q] = make_float2(f.x, f.y);
                v[2 * q + 1] = make_float2(f.z, f.w);
            }
#pragma unroll
            for (int c = 0; c < 2; c++) {
                float hu = 0.f, hv = 0.f, huu = 0.f, hvv = 0.f;
#pragma unroll
                for (int k = 0; k < K; k++) {
                    const float2 s = v[OFF + c + k];
                    const float gu = args.g[k] * s.x, gv = args.g[k] * s.y;
                    hu += gu;
                    hv += gv;
                    huu = fmaf(gu, s.x, huu);
                    hvv = fmaf(gv, s.y, hvv);
                }
                ring[c][t][0] = hu;
                ring[c][t][1] = hv;
                ring[c][t][2] = huu;
                ring[c][t][3] = hvv;
            }
            if (j >= 2 * R) {
                // vertical taps: output row i = j - 2R uses tile rows i .. i + 2R
                const int y = y0 + j - 2 * R;
                if (y < H) {
                    float wy;
                    if (y >= R && y < H - R) {
                        wy = gsum;
                    } else {
                        wy = 0.f;
#pragma unroll
                        for (int k = 0; k < K; k++) {
                            int yy = y + k - R;
                            wy += (yy >= 0 && yy < H) ? args.g[k] : 0.f;
                        }
                    }
#pragma unroll
                    for (int c = 0; c < 2; c++) {
                        float m[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                        for (int k = 0; k < K; k++) {
                            const int slot = (t + 1 + k) % K;
#pragma unroll
                            for (int q = 0; q < 4; q++) m[q] = fmaf(args.g[k], ring[c][slot][q], m[q]);
                        }
                        const int x = x0 + col0 + c;
                        if (x < W) {
                            const float inv = 1.0f / (wxv[c] * wy);
                            const float su = m[0] * inv, sv = m[1] * inv;  // shifted means
                            const float varu = m[2] * inv - su * su;
                            const float varv = m[3] * inv - sv * sv;
                            const float mu = su + cu, mv = sv + cv;
                            const float mu2 = mu * mu, mv2 = mv * mv;
                            const float num = (0.5f * (mu2 - mv2) + args.c1) * (0.5f * (varu - varv) + args.c2);
                            const float den = (0.5f * (mu2 + mv2) + args.c1) * (0.5f * (varu + varv) + args.c2);
                            const float ssim = num / den;
                            if (P.map) P.map[(long long)y * W + x] = ssim;
                            if (x >= pool_x_lo && x <= pool_x_hi && y >= pool_y_lo && y <= pool_y_hi) acc += ssim;
                        }
                    }
                }
            }
        }
    }

    // ---- deterministic pooling: CTA partial -> per-tile slot -> last CTA of the pair ----
    double d = double(acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_down_sync(0xffffffffu, d, o);
    if ((tid & 31) == 0) red[tid >> 5] = d;
    __syncthreads();
    if (tid == 0) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < NT / 32; i++) s += red[i];
        args.partials[gt] = s;
        __threadfence();
        unsigned prev = atomicAdd(&args.counters[pi], 1u);
        is_last = (prev == unsigned(P.ntiles - 1));
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    double s = 0.0;
    for (int i = tid; i < P.ntiles; i += NT) s += __ldcg(&args.partials[P.tile_base + i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __syncthreads();
    if ((tid & 31) == 0) red[tid >> 5] = s;
    __syncthreads();
    if (tid == 0) {
        double tot = 0.0;
#pragma unroll
        for (int i = 0; i < NT / 32; i++) tot += red[i];
        const double cnt = double(W - 2 * R + 1) * double(H - 2 * R + 1);
        args.scores[pi] = tot / cnt;
        args.counters[pi] = 0u;  // ready for the next launch
    }
}

template <int R>
void launch_ssim(const SsimArgs &a, int total_tiles, cudaStream_t s) {
    using G = Geom<R>;
    static bool attr_set = false;  // per process; the attribute is per device function
    if (!attr_set) {
        cudaFuncSetAttribute(ssim_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(G::SMEM));
        attr_set = true;
    }
    ssim_kernel<R><<<total_tiles, NT, G::SMEM, s>>>(a);
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
}

// Enqueue SSIM for device-resident pairs; `maps[i]` (device, nullable) receive the SSIM maps.
void ssim_enqueue(iqm_ctx *ctx, const std::vector<iqm_pair> &pairs, const iqm_ssim_params &p,
                  const std::vector<float *> &maps, double *d_scores) {
    const int n = int(pairs.size());
    const int R = (p.kernel_size - 1) / 2;
    const int S = strip_rows(R);
    std::vector<SsimPairDev> hd(n);
    int total = 0;
    for (int i = 0; i < n; i++) {
        const iqm_pair &q = pairs[i];
        SsimPairDev &d = hd[i];
        d.a = q.input;
        d.b = q.ref;
        d.map = maps.empty() ? nullptr : maps[i];
        d.pitch = (long long)q.row_bytes;
        d.w = q.w;
        d.h = q.h;
        d.tiles_x = int(iqm::ceil_div(q.w, TW));
        d.ntiles = d.tiles_x * int(iqm::ceil_div(q.h, S));
        d.tile_base = total;
        d.vec_ok = ((reinterpret_cast<uintptr_t>(q.input) | reinterpret_cast<uintptr_t>(q.ref) |
                     uintptr_t(q.row_bytes)) & 15u) == 0;
        total += d.ntiles;
    }
    auto *d_desc = static_cast<SsimPairDev *>(
        iqm::upload_bytes(ctx, ctx->desc, hd.data(), sizeof(SsimPairDev) * n));
    const size_t part_bytes = (sizeof(double) * total + 255) & ~size_t(255);
    const size_t cnt_bytes = (sizeof(unsigned) * n + 255) & ~size_t(255);
    auto *scr = static_cast<uint8_t *>(ctx->scratch.get(part_bytes + cnt_bytes, ctx->stream));
    SsimArgs a{};
    a.pairs = d_desc;
    a.npairs = n;
    a.partials = reinterpret_cast<double *>(scr);
    a.counters = reinterpret_cast<unsigned *>(scr + part_bytes);
    a.scores = d_scores;
    for (int k = 0; k < 15; k++) a.g[k] = 0.f;
    for (int k = -R; k <= R; k++) a.g[k + R] = float(std::exp(-double(k * k) / (2.0 * double(p.sigma) * p.sigma)));
    a.c1 = p.k1 * p.k1;
    a.c2 = p.k2 * p.k2;
    IQM_CHECK_CUDA(cudaMemsetAsync(a.counters, 0, sizeof(unsigned) * n, ctx->stream));
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
}

extern "C" __attribute__((visibility("default"))) int iqm_ssim_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n, const iqm_ssim_params *params,
                            double *d_scores) {
    return iqm::guarded(ctx, [&] {
        const iqm_ssim_params p = resolve(params);
        check_params(p);
        const int R = (p.kernel_size - 1) / 2;
        iqm::check_pairs(pairs, n, R, R);
        IQM_REQUIRE(d_scores != nullptr, "d_scores is NULL");
        ssim_enqueue(ctx, std::vector<iqm_pair>(pairs, pairs + n), p, {}, d_scores);
    });
}

extern "C" __attribute__((visibility("default"))) int iqm_ssim_batch(iqm_ctx *ctx, const iqm_pair *pairs, int n, const iqm_ssim_params *params,
                              double *scores) {
    return iqm::guarded(ctx, [&] {
        const iqm_ssim_params p = resolve(params);
        check_params(p);
        const int R = (p.kernel_size - 1) / 2;
        iqm::check_pairs(pairs, n, R, R);
        IQM_REQUIRE(scores != nullptr, "scores is NULL");
        auto dev = iqm::upload_pairs(ctx, pairs, n);
        auto *d_scores = static_cast<double *>(ctx->scores.get(sizeof(double) * n, ctx->stream));
        ssim_enqueue(ctx, dev, p, {}, d_scores);
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
