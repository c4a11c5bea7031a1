// FSIM / FSIMc on sm_100a.
//
// Reference path (cadik/IQM, src/gpu/fsim/fsim.cpp:80-163 and src/gpu/fsim/steps/*): downscale to
// W'xH' (F = max(1, round(min(W,H)/256))) as YIQ, gradient map, VkFFT forward transform of luma,
// 48 filtered spectra and 48 inverse transforms, per-orientation response sums, a host round trip
// for the noise medians, noise-energy estimates, phase congruency, similarity maps and three
// multi-pass float reductions.
//
// Here, per group of pairs with the same W'xH', seven kernels:
//   fsim_ingest_kernel      full-resolution RGBA8 -> I, Q, Y planes of both images (box F x F)
//   fsim_fwd_rows_kernel    forward FFT along x of a pair's two luma planes packed as one complex
//                           plane Y_img + i Y_ref (shared-memory Stockham)
//   fsim_fwd_cols_kernel    forward FFT along y
//   fsim_inv_cols_kernel    each image's spectrum separated from the packed one (Hermitian halves),
//                           x log-Gabor_s x angular_o, inverse FFT along y (32 planes)
//   fsim_inv_rows_kernel    inverse FFT along x of the 4 scales of one orientation, scaled 1/N,
//                           fused with the response sums of fsim_sum_filter_responses.glsl and
//                           the |EO(s=0)|^2 values of fsim_pack_for_median.glsl
//   fsim_noise_kernel       exact upper median by radix select (no host round trip), noise power
//                           and the phase-congruency threshold T in FP64
//   fsim_final_kernel       phase congruency, gradient (3x3 on the fly), similarity terms and the
//                           three pooled sums in FP64; the last CTA of a pair writes FSIM, FSIMc
// The 16 filters and the size-only constants (EM_n, EstSumAn2, EstSumAiAj; fsim_filter_noise.glsl,
// fsim_mult_filters.glsl) are built once per W'xH' with the same kernels and cached on the context.
// Schedule per group: ingest and the forward transform for all pairs at once; the two inverse passes
// in chunks of pairs whose 32 intermediate planes fit the 126 MB L2; noise and final kernels for
// all pairs at once.  Every transform runs on one warp (fft.cuh warp engine), CTAs hold 1-8 of
// them, so stages synchronise with __syncwarp only.
#include <algorithm>
#include <cmath>
#include <initializer_list>
#include <map>
#include <mutex>
#include <tuple>

#include "dft_mma.cuh"
#include "fft.cuh"
#include "fft_plan.cuh"
#include "iqm_internal.cuh"
#include "select.cuh"

#define GLSL_PI 3.141592653589

namespace iqm {

struct FsimPlan {
    int w2 = 0, h2 = 0, n = 0;
    FftLen row{}, col{};
    float *filters = nullptr;  // 16 planes of n (z = o*4 + s)
    double *consts = nullptr;  // device: em[4], an2[2][4], aiaj[2][4]
    void *mma_tables = nullptr;  // tensor-core engines' constants (480 x 270 plans in a mixed form)
    double em[4], an2[2][4], aiaj[2][4];
    ~FsimPlan() {
        if (filters) cudaFree(filters);
        if (consts) cudaFree(consts);
        if (mma_tables) cudaFree(mma_tables);
    }
};

}  // namespace iqm

using iqm::FftLen;

namespace {

constexpr int FT = 256;  // threads per FFT / pointwise CTA

struct FsimPairDev {
    const uint8_t *a;
    const uint8_t *b;
    long long pitch;
    int w, h, F;
    int out;  // index of this pair in the caller's score array
};

struct FsimGroup {
    const FsimPairDev *pairs;
    int G;          // pairs in this launch
    int pair0;      // group index of the first pair of this launch (inverse-pass chunks)
    int w2, h2, n;
    float *yiq;     // G x 2 x 3 x n   (I, Q, Y)
    float2 *spec;   // G x n: per pair the spectrum of Y_img + i Y_ref
    float2 *T;      // chunk x 2 x 16 x n  (after the column pass of the inverse transform)
    __half2 *Th;    // the same planes in FP16 (mixed precision; shares T's memory)
    float *amp;     // G x 8 x n       (img*4 + o)
    float *energy;  // G x 8 x n
    float *eo0;     // G x 8 x n       |EO(s=0, o)|^2
    float *thr;     // G x 8
    double *partials;  // G x tiles x 3
    unsigned *counters;
    int tiles;
    double *scores;    // 2 per pair: fsim, fsimc
    const float *filters;  // 16 planes, column-major: filters[z][x * h2 + y]
    const double *consts;
    int energy_mode;
};

// ---------------------------------------------------------------------------------------------
// filters -- shaders/fsim/fsim_lowpassfilter.glsl:21-42 (cutoff 0.45, order 15),
// fsim_log_gabor.glsl:16-49 (minWaveLength 6, mult 2, sigmaOnf 0.55), fsim_angular.glsl:16-48,
// combined as in fsim_filter_combinations.glsl:44-51 (z = o*4 + s)
__device__ __forceinline__ float freq_coord(int i, int n) {
    const int shifted = (i + n / 2) % n;
    return float(shifted - n / 2) / float(n);
}

__global__ void fsim_filters_kernel(float *filters, int w2, int h2) {
    const int n = w2 * h2;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int x = p % w2, y = p / w2;
    const float sx = freq_coord(x, w2), sy = freq_coord(y, h2);
    const float radius = sqrtf(sx * sx + sy * sy);
    const float lp = 1.0f / (1.0f + powf(radius / 0.45f, 2.0f * 15.0f));
    float lg[4];
#pragma unroll
    for (int s = 0; s < 4; s++) {
        const float wavelength = 6.0f * powf(2.0f, float(s));
        const float freq = 1.0f / wavelength;
        const float lr = logf(radius / freq);
        const float ls = logf(0.55f);
        const float v = expf(-(lr * lr) / (2.0f * (ls * ls)));
        lg[s] = (x == 0 && y == 0) ? 0.0f : v * lp;
    }
    const float theta_sigma = float(GLSL_PI) / 4.0f / 1.2f;
    const float theta = atan2f(-sy, sx);
    const float st = sinf(theta), ct = cosf(theta);
#pragma unroll
    for (int o = 0; o < 4; o++) {
        const float angle = (float(o) * float(GLSL_PI)) / 4.0f;
        const float ds = st * cosf(angle) - ct * sinf(angle);
        const float dc = ct * cosf(angle) + st * sinf(angle);
        const float dtheta = fabsf(atan2f(ds, dc));
        const float a = expf(-(dtheta * dtheta) / (2.0f * (theta_sigma * theta_sigma)));
#pragma unroll
        for (int s = 0; s < 4; s++) filters[(o * 4 + s) * n + x * h2 + y] = lg[s] * a;
    }
}

// EM_n(o) = sum_p H[o*4+0](p)^2 (fsim_filter_combinations.cpp:76-134 with fsim_filter_noise.glsl)
__global__ void fsim_em_kernel(const float *filters, int n, double *consts) {
    __shared__ double red[FT / 32];
    const int o = blockIdx.x;
    const float *f = filters + (o * 4) * n;
    double s = 0.0;
    for (int p = threadIdx.x; p < n; p += FT) {
        const float v = f[p];
        s += double(v * v);
    }
    for (int d = 16; d > 0; d >>= 1) s += __shfl_down_sync(0xffffffffu, s, d);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < FT / 32; i++) t += red[i];
        consts[o] = t;
    }
}

// ---------------------------------------------------------------------------------------------
// ingest -- shaders/fsim/fsim_downsample.glsl:21-55: RGB x 255 -> (I, Q, Y), F x F box starting
// at (x F - F/2, y F - F/2), out-of-image samples contribute 0, divided by F^2 always.
// The shader's unorm load followed by x 255 gives back the byte value exactly in FP32
// ((b / 255) * 255 == b for every byte b), and the YIQ transform is linear, so each window's channel
// bytes are summed as integers (exact) and transformed once; the shader's per-sample FP32
// accumulation differs from this only by its own rounding.
template <int FF>  // FF = downscale factor when known at compile time, 0 = read it from the pair
__global__ void __launch_bounds__(FT) fsim_ingest_kernel(FsimGroup g) {
    const int pi = blockIdx.y;
    const int p = blockIdx.x * FT + threadIdx.x;
    if (p >= g.n) return;
    const FsimPairDev P = g.pairs[pi];
    const int x = p % g.w2, y = p / g.w2;
    const int F = FF ? FF : P.F;
    const int xs = x * F - F / 2, ys = y * F - F / 2;
    const float scaler = float(F * F);
    unsigned rb[2] = {0u, 0u}, gs[2] = {0u, 0u};  // FF != 0: R | B << 16 per image (F^2 * 255 < 2^16)
    unsigned r32[2] = {0u, 0u}, b32[2] = {0u, 0u};  // FF == 0: R and B of a window of any size
    if constexpr (FF == 4 || FF == 8) {
        // the window's F pixels of a row start at byte 4F x - 2F: 8-byte aligned for F = 4,
        // 16-byte aligned for F = 8 (given an aligned base and pitch); rows load as vectors when
        // the whole row is inside the image
        constexpr int V = FF == 4 ? 2 : 4;  // pixels per vector load
#pragma unroll
        for (int img = 0; img < 2; img++) {
            const uint8_t *base = img ? P.b : P.a;
            const bool vec = ((reinterpret_cast<uintptr_t>(base) | uintptr_t(P.pitch)) & (4 * V - 1)) == 0 &&
                             xs >= 0 && xs + FF <= P.w;
#pragma unroll
            for (int kk = 0; kk < FF; kk++) {
                const int k = ys + kk;
                if (k < 0 || k >= P.h) continue;
                const uint32_t *row = reinterpret_cast<const uint32_t *>(base + (long long)k * P.pitch);
                uint32_t px[FF];
                if (vec) {
#pragma unroll
                    for (int q = 0; q < FF / V; q++) {
                        if constexpr (V == 2) {
                            const uint2 t = __ldg(reinterpret_cast<const uint2 *>(row + xs) + q);
                            px[2 * q] = t.x;
                            px[2 * q + 1] = t.y;
                        } else {
                            const uint4 t = __ldg(reinterpret_cast<const uint4 *>(row + xs) + q);
                            px[4 * q] = t.x;
                            px[4 * q + 1] = t.y;
                            px[4 * q + 2] = t.z;
                            px[4 * q + 3] = t.w;
                        }
                    }
                } else {
#pragma unroll
                    for (int jj = 0; jj < FF; jj++) {
                        const int j = xs + jj;
                        px[jj] = (j >= 0 && j < P.w) ? __ldg(row + j) : 0u;
                    }
                }
#pragma unroll
                for (int jj = 0; jj < FF; jj++) {
                    rb[img] += px[jj] & 0x00ff00ffu;
                    gs[img] += (px[jj] >> 8) & 0xffu;
                }
            }
        }
    } else {
#pragma unroll
        for (int img = 0; img < 2; img++) {
            const uint8_t *base = img ? P.b : P.a;
            for (int kk = 0; kk < F; kk++) {
                const int k = ys + kk;
                if (k < 0 || k >= P.h) continue;
                const uint32_t *row = reinterpret_cast<const uint32_t *>(base + (long long)k * P.pitch);
                for (int jj = 0; jj < F; jj++) {
                    const int j = xs + jj;
                    if (j < 0 || j >= P.w) continue;
                    const uint32_t v = __ldg(row + j);
                    if constexpr (FF == 0) {
                        r32[img] += v & 0xffu;
                        b32[img] += (v >> 16) & 0xffu;
                    } else {
                        rb[img] += v & 0x00ff00ffu;
                    }
                    gs[img] += (v >> 8) & 0xffu;
                }
            }
        }
    }
#pragma unroll
    for (int img = 0; img < 2; img++) {
        const float r = float(FF ? rb[img] & 0xffffu : r32[img]);
        const float b = float(FF ? rb[img] >> 16 : b32[img]);
        const float gg = float(gs[img]);
        float *dst = g.yiq + size_t(pi * 2 + img) * 3 * g.n;
        dst[p] = (r * 0.596f - gg * 0.274f - b * 0.322f) / scaler;
        dst[g.n + p] = (r * 0.211f - gg * 0.523f + b * 0.312f) / scaler;
        dst[2 * g.n + p] = (r * 0.299f + gg * 0.587f + b * 0.114f) / scaler;
    }
}

// ---------------------------------------------------------------------------------------------
// Transform kernels.  Shared memory of every transform CTA starts with the stage twiddles of its
// length (FftLen::stw), followed by per-warp work buffers: a warp transforms NB sequences at once in
// buffer a (NB x wl) and, unless the engine transforms in place, a ping-pong buffer b of the same
// size.
constexpr int NB = 1;  // the transform engines run one sequence per warp
static_assert(NB == 1, "column slabs index with cols == 1 << lw");


// Transform engines: the runtime-planned warp engine for any length, or a fixed-length one whose
// radix sequence is compiled in (the host picks it only when it equals the length's own plan, so
// the stage twiddle table in shared memory has the layout it expects).
struct GenericEngine {
    static __device__ __forceinline__ float2 *run(float2 *a, float2 *b, const FftLen &L, const float2 *stw, float s,
                                                  int wl) {
        return iqm::fft_warp(a, b, L, stw, s, 1, wl);
    }
};
template <class FP>
struct FixedEngine {
    static __device__ __forceinline__ float2 *run(float2 *a, float2 *b, const FftLen &, const float2 *stw, float s,
                                                  int) {
        return FP::run(a, b, stw, s);
    }
};
// Transform length an engine is compiled for (0: any length).
template <class E>
struct engine_len {
    static constexpr int value = 0;
};
template <class FP>
struct engine_len<FixedEngine<FP>> {
    static constexpr int value = FP::n;
};

// Work buffers a transform needs: two for the ping-pong engines, one for the in-place fixed plans.
template <class FP>
struct plan_bufs {
    static constexpr int value = 2;
};
template <int N, int... Rs>
struct plan_bufs<iqm::FixedPlanIP<N, Rs...>> {
    static constexpr int value = 1;
};
template <class E>
struct engine_bufs {
    static constexpr int value = 2;
};
template <class FP>
struct engine_bufs<FixedEngine<FP>> {
    static constexpr int value = plan_bufs<FP>::value;
};

// The work area of warp `warp` in a CTA whose warps each hold engine_bufs<E> buffers of wl points.
template <class E>
__device__ __forceinline__ float2 *warp_area(float2 *base, int warp, int wl) {
    return base + size_t(warp) * engine_bufs<E>::value * NB * wl;
}

// 480 (the row length, whose pass is limited by shared memory) transforms in place; 270 (the column
// length, whose pass is limited by registers) keeps the two-buffer form.
using Engine270 = FixedEngine<iqm::FixedPlan<270, 9, 3, 10>>;
using Engine480 = FixedEngine<iqm::FixedPlanIP<480, 15, 8, 4>>;

// Strided copy with up to 8 independent loads in flight per thread: ld(i) for i = first, first +
// step, ... < n, in batches of 8 loads before their 8 stores st(i, v) (runtime-length paths, whose
// plain loops would wait for each load before issuing the next).
template <class T, class Ld, class St>
__device__ __forceinline__ void batched_copy(int first, int n, int step, Ld ld, St st) {
    for (int i0 = first; i0 < n; i0 += 8 * step) {
        T v[8];
#pragma unroll
        for (int k = 0; k < 8; k++)
            if (i0 + k * step < n) v[k] = ld(i0 + k * step);
#pragma unroll
        for (int k = 0; k < 8; k++)
            if (i0 + k * step < n) st(i0 + k * step, v[k]);
    }
}
struct F2x2 {
    float2 z, m;
};

// forward transform (src/gpu/fsim/fsim.cpp:270-368: luma as complex (Y, 0), sign -1, unscaled),
// NB rows per warp.
template <class Eng>
// Compiled engines: 4 CTAs per SM (62 registers with the 480-point engine, no spills).
__global__ void __launch_bounds__(FT, engine_len<Eng>::value ? 4 : 1) fsim_fwd_rows_kernel(FsimGroup g, const __grid_constant__ FftLen L, int wl) {
    extern __shared__ __align__(16) float2 sm[];
    const int tl = iqm::stage_twiddle_len(L);
    iqm::stage_twiddles_to_shared(L, sm);
    __syncthreads();
    float2 *work = sm + ((tl + 1) & ~1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // the two real luma planes of a pair transform together as one complex plane Y_img + i Y_ref
    const int pair = blockIdx.y;
    const int y0 = (blockIdx.x * (blockDim.x >> 5) + warp) * NB;
    if (y0 >= g.h2) return;  // warp-uniform; no block-wide barrier follows
    const int nb = min(NB, g.h2 - y0);
    float2 *a = warp_area<Eng>(work, warp, wl), *b = a + NB * wl;
    const float *Y1 = g.yiq + (size_t(pair * 2) * 3 + 2) * g.n + size_t(y0) * g.w2;
    const float *Y2 = Y1 + size_t(3) * g.n;  // the pair's second image
    constexpr int PN = engine_len<Eng>::value;
    for (int t = 0; t < nb; t++) {
        if constexpr (PN > 0) {  // fixed length: the row's loads all in flight before the stores
            constexpr int PV = (PN + 31) / 32;
            float v1[PV], v2[PV];
#pragma unroll
            for (int i = 0; i < PV; i++)
                if (lane + 32 * i < PN) {
                    v1[i] = __ldcg(Y1 + size_t(t) * g.w2 + lane + 32 * i);
                    v2[i] = __ldcg(Y2 + size_t(t) * g.w2 + lane + 32 * i);
                }
#pragma unroll
            for (int i = 0; i < PV; i++)
                if (lane + 32 * i < PN) a[t * wl + lane + 32 * i] = make_float2(v1[i], v2[i]);
        } else {
            batched_copy<float2>(
                lane, g.w2, 32, [&](int x) { return make_float2(Y1[size_t(t) * g.w2 + x], Y2[size_t(t) * g.w2 + x]); },
                [&](int x, float2 v) { a[t * wl + x] = v; });
        }
    }
    const float2 *res = Eng::run(a, b, L, sm, -1.f, wl);
    float2 *S = g.spec + size_t(pair) * g.n + size_t(y0) * g.w2;
    for (int t = 0; t < nb; t++)
        for (int x = lane; x < g.w2; x += 32) S[size_t(t) * g.w2 + x] = res[t * wl + x];
}

// Column passes: a CTA of nw warps owns NB*nw adjacent columns (nw power of two); the column slab
// is loaded and stored cooperatively and each warp transforms NB of its columns.
__device__ __forceinline__ int slab_parity(float2 *res, float2 *a) { return res == a ? 0 : 1; }

template <class Eng>
// Compiled engines: 5 CTAs per SM with the two-buffer 270-point engine (48 registers), 4 with the
// in-place 480-point one (63 registers); no spills either way.
__global__ void __launch_bounds__(FT, engine_len<Eng>::value ? (engine_bufs<Eng>::value == 2 ? 5 : 4) : 1)
fsim_fwd_cols_kernel(FsimGroup g, const __grid_constant__ FftLen L, int wl, int lw) {
    extern __shared__ __align__(16) float2 sm[];
    __shared__ int parity;
    const int tl = iqm::stage_twiddle_len(L);
    iqm::stage_twiddles_to_shared(L, sm);
    float2 *work = sm + ((tl + 1) & ~1);
    const int nw = 1 << lw, cols = NB * nw, warp = threadIdx.x >> 5;
    const int pair = blockIdx.y;
    const int x0 = blockIdx.x * cols;
    const int nc = min(cols, g.w2 - x0);
    float2 *S = g.spec + size_t(pair) * g.n;
    // column c lives in warp c / NB, slot c % NB
    constexpr int PN = engine_len<Eng>::value;
    if constexpr (PN > 0) {  // fixed length: each thread's slab loads all in flight before the stores
        constexpr int KS = (NB * PN + 31) / 32;
        float2 v[KS];
#pragma unroll
        for (int k = 0; k < KS; k++) {
            const int idx = threadIdx.x + k * blockDim.x;
            const int c = idx & (cols - 1), y = idx >> lw;  // cols = 1 << lw
            if (idx < cols * g.h2 && c < nc) v[k] = __ldcg(S + size_t(y) * g.w2 + x0 + c);
        }
#pragma unroll
        for (int k = 0; k < KS; k++) {
            const int idx = threadIdx.x + k * blockDim.x;
            const int c = idx & (cols - 1), y = idx >> lw;
            if (idx < cols * g.h2 && c < nc) warp_area<Eng>(work, c / NB, wl)[(c % NB) * wl + y] = v[k];
        }
    } else {
        batched_copy<float2>(
            threadIdx.x, cols * g.h2, blockDim.x,
            [&](int idx) {
                const int c = idx & (cols - 1), y = idx >> lw;  // cols = 1 << lw
                return c < nc ? S[size_t(y) * g.w2 + x0 + c] : make_float2(0.f, 0.f);
            },
            [&](int idx, float2 v) {
                const int c = idx & (cols - 1), y = idx >> lw;
                if (c < nc) warp_area<Eng>(work, c / NB, wl)[(c % NB) * wl + y] = v;
            });
    }
    __syncthreads();
    const int nbw = min(NB, nc - warp * NB);
    if (nbw > 0) {
        float2 *a = warp_area<Eng>(work, warp, wl);
        float2 *res = Eng::run(a, a + NB * wl, L, sm, -1.f, wl);
        if (warp == 0 && (threadIdx.x & 31) == 0) parity = slab_parity(res, a);
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < cols * g.h2; idx += blockDim.x) {
        const int c = idx & (cols - 1), y = idx >> lw;  // cols = 1 << lw
        if (c < nc) S[size_t(y) * g.w2 + x0 + c] = warp_area<Eng>(work, c / NB, wl)[parity * NB * wl + (c % NB) * wl + y];
    }
}

// ---------------------------------------------------------------------------------------------
// inverse transform, pass 1 (along y) of the 4 filtered spectra of orientation o:
// spectrum x H[o*4+s] (fsim_filter_combinations.glsl:53-56), sign +1.  consts_mode uses a
// spectrum of ones, i.e. transforms the filters themselves (block 0 of the reference's buffer).
template <class Eng>
// Two-buffer compiled engines: 4 CTAs per SM (64 registers; with the largest shared-memory carveout
// the work buffers of 4 CTAs fit).  The runtime-planned and in-place engines need more registers here.
__global__ void __launch_bounds__(FT, engine_len<Eng>::value && engine_bufs<Eng>::value == 2 ? 4 : 1)
fsim_inv_cols_kernel(FsimGroup g, const __grid_constant__ FftLen L, int wl, int lw, int consts_mode) {
    extern __shared__ __align__(16) float2 sm[];
    __shared__ int parity;
    const int tl = iqm::stage_twiddle_len(L);
    iqm::stage_twiddles_to_shared(L, sm);
    const int nw = 1 << lw, cols = NB * nw, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int o = blockIdx.y;
    const int plane = blockIdx.z;  // chunk-local pair*2 + img
    const int x0 = blockIdx.x * cols;
    const int nc = min(cols, g.w2 - x0);
    const int h2 = g.h2;
    float2 *Sl = sm + ((tl + 1) & ~1);     // cols x h2 spectrum slab (column-major)
    float2 *work = Sl + size_t(cols) * h2;  // per warp: a, b of NB x wl each
    const int img = plane & 1;
    const float2 *src = g.spec + size_t(g.pair0 + (plane >> 1)) * g.n;  // the pair's packed spectrum
    const int nbw = min(NB, nc - warp * NB);
    // With a fixed-length engine (h2 == PN) each lane holds its share of the warp's filter column in
    // registers, and the next scale's share is loaded while this scale's transform runs.
    constexpr int PN = engine_len<Eng>::value;
    constexpr int PV = PN > 0 ? (PN + 31) / 32 : 1;
    float hnext[PV];
    auto load_filter = [&](int zz) {
        const float *H = g.filters + size_t(zz) * g.n + size_t(x0 + warp) * h2;
#pragma unroll
        for (int i = 0; i < PV; i++) {
            const int y = lane + 32 * i;
            hnext[i] = (y < PN) ? __ldg(H + y) : 0.f;
        }
    };
    if (PN > 0 && nbw > 0) load_filter(o * 4);
    // Z = F(Y_img + i Y_ref): F(Y_img) = (Z(k) + conj Z(-k)) / 2, F(Y_ref) = (Z(k) - conj Z(-k)) / 2i
    auto separate = [&](float2 z, float2 m) {
        return img == 0 ? make_float2(0.5f * (z.x + m.x), 0.5f * (z.y - m.y))
                        : make_float2(0.5f * (z.y + m.y), 0.5f * (m.x - z.x));
    };
    if constexpr (PN > 0) {
        // fixed length: each thread's NB * PN / 32 slab entries, all loads in flight before the stores
        // (blockDim.x = 32 nw threads cover cols * PN = NB nw PN entries)
        constexpr int KS = (NB * PN + 31) / 32;
        float2 zv[KS], mv[KS];
#pragma unroll
        for (int k = 0; k < KS; k++) {
            const int idx = threadIdx.x + k * blockDim.x;
            const int c = idx & (cols - 1), y = idx >> lw;  // cols = 1 << lw
            zv[k] = mv[k] = make_float2(1.f, 0.f);
            if (idx < cols * h2 && c < nc && !consts_mode) {
                const int x = x0 + c;
                zv[k] = __ldcg(src + size_t(y) * g.w2 + x);
                mv[k] = __ldcg(src + size_t(y ? h2 - y : 0) * g.w2 + (x ? g.w2 - x : 0));
            }
        }
#pragma unroll
        for (int k = 0; k < KS; k++) {
            const int idx = threadIdx.x + k * blockDim.x;
            const int c = idx & (cols - 1), y = idx >> lw;
            if (idx < cols * h2 && c < nc) Sl[size_t(c) * h2 + y] = consts_mode ? make_float2(1.f, 0.f) : separate(zv[k], mv[k]);
        }
    } else {
        batched_copy<F2x2>(
            threadIdx.x, cols * h2, blockDim.x,
            [&](int idx) {
                const int c = idx & (cols - 1), y = idx >> lw;  // cols = 1 << lw
                F2x2 p{make_float2(1.f, 0.f), make_float2(1.f, 0.f)};
                if (c < nc && !consts_mode) {
                    const int x = x0 + c;
                    p.z = src[size_t(y) * g.w2 + x];
                    p.m = src[size_t(y ? h2 - y : 0) * g.w2 + (x ? g.w2 - x : 0)];
                }
                return p;
            },
            [&](int idx, F2x2 p) {
                const int c = idx & (cols - 1), y = idx >> lw;
                if (c < nc) Sl[size_t(c) * h2 + y] = consts_mode ? make_float2(1.f, 0.f) : separate(p.z, p.m);
            });
    }
    __syncthreads();
    for (int s = 0; s < 4; s++) {
        const int z = o * 4 + s;
        if (nbw > 0) {
            float2 *a = warp_area<Eng>(work, warp, wl);
            const float2 *col = Sl + size_t(warp) * h2;  // NB == 1: column `warp` of the slab
            if constexpr (PN > 0) {
                float hcur[PV];
#pragma unroll
                for (int i = 0; i < PV; i++) hcur[i] = hnext[i];
                if (s < 3) load_filter(z + 1);
#pragma unroll
                for (int i = 0; i < PV; i++) {
                    const int y = lane + 32 * i;
                    if (y < PN) {
                        const float2 v = col[y];
                        a[y] = make_float2(hcur[i] * v.x, hcur[i] * v.y);
                    }
                }
            } else {
                const float *H = g.filters + size_t(z) * g.n + size_t(x0 + warp) * h2;
                for (int y = lane; y < h2; y += 32) {
                    const float hv = __ldg(H + y);
                    const float2 v = col[y];
                    a[y] = make_float2(hv * v.x, hv * v.y);
                }
            }
            float2 *res = Eng::run(a, a + NB * wl, L, sm, 1.f, wl);
            if (warp == 0 && lane == 0) parity = slab_parity(res, a);
        }
        __syncthreads();
        float2 *dst = g.T + (size_t(plane) * 16 + z) * g.n;
        for (int idx = threadIdx.x; idx < cols * h2; idx += blockDim.x) {
            const int c = idx & (cols - 1), y = idx >> lw;  // cols = 1 << lw
            if (c < nc) dst[size_t(y) * g.w2 + x0 + c] = warp_area<Eng>(work, c / NB, wl)[parity * NB * wl + (c % NB) * wl + y];
        }
        __syncthreads();
    }
}

// CTA-wide form of the inverse column pass for long columns (runtime-planned lengths whose per-warp
// work buffers would leave few warps per SM): the whole CTA transforms `cb` adjacent columns at once
// with the block-level engine, one scale after another; the cb-column slab keeps the global loads and
// stores in row segments.
__global__ void __launch_bounds__(FT, 1)
fsim_inv_cols_seq_kernel(FsimGroup g, const __grid_constant__ FftLen L, int wl, int cb) {
    extern __shared__ __align__(16) float2 sm[];
    const int o = blockIdx.y;
    const int plane = blockIdx.z;  // chunk-local pair*2 + img
    const int img = plane & 1;
    const int w2 = g.w2, h2 = g.h2;
    const int x0 = blockIdx.x * cb;
    const int nc = min(cb, w2 - x0);
    float2 *Sl = sm;                   // nc x h2 separated spectrum (column-major)
    float2 *a = Sl + size_t(cb) * h2;  // nc x wl
    float2 *b = a + size_t(cb) * wl;   // nc x wl
    const float2 *src = g.spec + size_t(g.pair0 + (plane >> 1)) * g.n;  // the pair's packed spectrum
    batched_copy<F2x2>(
        threadIdx.x, nc * h2, blockDim.x,
        [&](int idx) {
            const int y = idx / nc, c = idx - y * nc;
            const int x = x0 + c;
            return F2x2{src[size_t(y) * w2 + x], src[size_t(y ? h2 - y : 0) * w2 + (x ? w2 - x : 0)]};
        },
        [&](int idx, F2x2 p) {
            const int y = idx / nc, c = idx - y * nc;
            const float2 z = p.z, m = p.m;
            Sl[size_t(c) * h2 + y] = img == 0 ? make_float2(0.5f * (z.x + m.x), 0.5f * (z.y - m.y))
                                              : make_float2(0.5f * (z.y + m.y), 0.5f * (m.x - z.x));
        });
    __syncthreads();
    for (int s = 0; s < 4; s++) {
        const int z = o * 4 + s;
        const float *H = g.filters + size_t(z) * g.n + size_t(x0) * h2;  // column-major filter plane
        batched_copy<float>(
            threadIdx.x, nc * h2, blockDim.x, [&](int idx) { return __ldg(H + idx); },
            [&](int idx, float hv) {
                const int c = idx / h2, y = idx - c * h2;
                const float2 v = Sl[idx];
                a[size_t(c) * wl + y] = make_float2(hv * v.x, hv * v.y);
            });
        __syncthreads();
        const float2 *res = iqm::fft_run(a, b, L, 1.f, nc, wl);
        float2 *dst = g.T + (size_t(plane) * 16 + z) * g.n;
        for (int idx = threadIdx.x; idx < nc * h2; idx += blockDim.x) {
            const int y = idx / nc, c = idx - y * nc;
            dst[size_t(y) * w2 + x0 + c] = res[size_t(c) * wl + y];
        }
        __syncthreads();
    }
}

// Per-pixel response sums of one orientation from its 4 scales (scaled by 1/N here), as
// shaders/fsim/fsim_sum_filter_responses.glsl:43-80 and fsim_pack_for_median.glsl:39-43; square
// roots and the reciprocal from the SFU approximations.
__device__ __forceinline__ void response_sums(const float2 v[4], float invN, float &sA, float &en, float &e0) {
    float re[4], im[4];
    float sE = 0.f, sO = 0.f;
    sA = 0.f;
#pragma unroll
    for (int s = 0; s < 4; s++) {
        re[s] = v[s].x * invN;
        im[s] = v[s].y * invN;
        sA += iqm::sqrt_nonneg(re[s] * re[s] + im[s] * im[s]);
        sE += re[s];
        sO += im[s];
    }
    const float rxe = iqm::rcp_approx(iqm::sqrt_nonneg(sE * sE + sO * sO) + 0.0001f);
    const float mE = sE * rxe, mO = sO * rxe;
    en = 0.f;
#pragma unroll
    for (int s = 0; s < 4; s++) en += re[s] * mE + im[s] * mO - fabsf(re[s] * mO - im[s] * mE);
    e0 = re[0] * re[0] + im[0] * im[0];
}

// inverse transform, pass 2 (along x): a CTA handles rr rows with WPR = 4/NB warps per row;
// warp (r, h) transforms scales h*NB .. h*NB+NB-1 of row y0 + r.  consts_mode (rr = 1) instead accumulates, per row, sum_s Re_s^2 N and
// sum_{i<j} Re_i Re_j N (shaders/fsim/fsim_mult_filters.glsl:37-58) over p < ceil(N/2) and all p.
template <class Eng>
__global__ void __launch_bounds__(FT, engine_len<Eng>::value ? 4 : 1) fsim_inv_rows_kernel(FsimGroup g, const __grid_constant__ FftLen L, int wl, int rr, int consts_mode,
                                                              double *rowsums) {
    extern __shared__ __align__(16) float2 sm[];
    __shared__ int parity;
    __shared__ double red[4][FT / 32];
    const int tl = iqm::stage_twiddle_len(L);
    iqm::stage_twiddles_to_shared(L, sm);
    __syncthreads();
    float2 *work = sm + ((tl + 1) & ~1);
    constexpr int WPR = 4 / NB;  // warps per row
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = warp / WPR, h = warp % WPR;
    const int o = blockIdx.y, plane = blockIdx.z;  // plane: chunk-local pair*2 + img
    const int w2 = g.w2;
    const int y0 = blockIdx.x * rr;
    {
        const int y = y0 + r;
        if (r < rr && y < g.h2) {
            float2 *a = warp_area<Eng>(work, warp, wl);
            constexpr int PN = engine_len<Eng>::value;
            for (int t = 0; t < NB; t++) {
                const float2 *src = g.T + (size_t(plane) * 16 + o * 4 + h * NB + t) * g.n + size_t(y) * w2;
                if constexpr (PN > 0) {
                    // fixed length: every load of the row is in flight before the first store
                    constexpr int PV = (PN + 31) / 32;
                    float2 v[PV];
#pragma unroll
                    for (int i = 0; i < PV; i++)
                        if (lane + 32 * i < PN) v[i] = __ldcg(src + lane + 32 * i);
#pragma unroll
                    for (int i = 0; i < PV; i++)
                        if (lane + 32 * i < PN) a[t * wl + lane + 32 * i] = v[i];
                } else {
                    batched_copy<float2>(lane, w2, 32, [&](int x) { return src[x]; },
                                         [&](int x, float2 v) { a[t * wl + x] = v; });
                }
            }
            float2 *res = Eng::run(a, a + NB * wl, L, sm, 1.f, wl);
            if (warp == 0 && lane == 0) parity = slab_parity(res, a);
        }
    }
    __syncthreads();
    // scale s of row rl: warp rl*WPR + s/NB, slot s%NB
    auto at = [&](int rl, int s, int x) -> float2 {
        return warp_area<Eng>(work, rl * WPR + s / NB, wl)[parity * NB * wl + (s % NB) * wl + x];
    };
    const float invN = 1.0f / float(g.n);
    if (!consts_mode && (w2 & 3) == 0 && rr <= 2) {
        // 4 consecutive pixels a thread: 16-byte reads of each scale's result, 16-byte stores (rows
        // of w2 % 4 == 0 pixels keep every quad aligned: plane sizes and row offsets are multiples of 4)
        const int gp = g.pair0 * 2 + plane;
        const int qpr = w2 >> 2;  // quads per row
        for (int idx = threadIdx.x; idx < rr * qpr; idx += blockDim.x) {
            const int rl = idx >= qpr ? 1 : 0;
            const int x = (idx - rl * qpr) * 4;
            const int y = y0 + rl;
            if (y >= g.h2) continue;
            float4 oa, oe, o0;
            float *pa = &oa.x, *pe = &oe.x, *p0 = &o0.x;
            float2 v[4][4];  // [scale][pixel]
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float4 *src4 = reinterpret_cast<const float4 *>(&warp_area<Eng>(work, rl * WPR + q / NB, wl)[parity * NB * wl + (q % NB) * wl + x]);
                const float4 lo = src4[0], hi = src4[1];
                v[q][0] = make_float2(lo.x, lo.y);
                v[q][1] = make_float2(lo.z, lo.w);
                v[q][2] = make_float2(hi.x, hi.y);
                v[q][3] = make_float2(hi.z, hi.w);
            }
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const float2 w[4] = {v[0][i], v[1][i], v[2][i], v[3][i]};
                response_sums(w, invN, pa[i], pe[i], p0[i]);
            }
            const size_t off = (size_t(gp) * 4 + o) * g.n + size_t(y) * w2 + x;
            *reinterpret_cast<float4 *>(g.amp + off) = oa;
            *reinterpret_cast<float4 *>(g.energy + off) = oe;
            *reinterpret_cast<float4 *>(g.eo0 + off) = o0;
        }
    } else if (!consts_mode) {
        const int gp = g.pair0 * 2 + plane;
        for (int rl = 0; rl < rr; rl++) {
            const int y = y0 + rl;
            if (y >= g.h2) break;
            const size_t row = (size_t(gp) * 4 + o) * g.n + size_t(y) * w2;
            for (int x = threadIdx.x; x < w2; x += blockDim.x) {
                float2 v[4];
#pragma unroll
                for (int q = 0; q < 4; q++) v[q] = at(rl, q, x);
                float sA, en, e0;
                response_sums(v, invN, sA, en, e0);
                g.amp[row + x] = sA;
                g.energy[row + x] = en;
                g.eo0[row + x] = e0;
            }
        }
    } else {
        const int y = y0;  // rr == 1
        const long lim = (long(g.n) + 1) / 2;
        const float fn = float(g.n);
        double acc[4] = {0.0, 0.0, 0.0, 0.0};  // an2 (ref), aiaj (ref), an2 (full), aiaj (full)
        for (int x = threadIdx.x; x < w2; x += blockDim.x) {
            float re[4];
#pragma unroll
            for (int q = 0; q < 4; q++) re[q] = at(0, q, x).x * invN;
            float q2 = 0.f, qx = 0.f;
#pragma unroll
            for (int q = 0; q < 4; q++) q2 += (re[q] * re[q]) * fn;
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = i + 1; j < 4; j++) qx += re[i] * re[j] * fn;
            const long p = long(y) * w2 + x;
            if (p < lim) {
                acc[0] += q2;
                acc[1] += qx;
            }
            acc[2] += q2;
            acc[3] += qx;
        }
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            double v = acc[q];
            for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
            if (lane == 0) red[q][warp] = v;
        }
        __syncthreads();
        if (threadIdx.x < 4) {
            double t = 0.0;
            for (int i = 0; i < nw; i++) t += red[threadIdx.x][i];
            rowsums[(size_t(o) * g.h2 + y) * 4 + threadIdx.x] = t;
        }
    }
}

// Sequential form of pass 2 for rows too long for four warp buffers (Bluestein lengths): the whole
// CTA transforms `sb` scales at a time (1, 2 or 4) with the block-level engine.
__global__ void __launch_bounds__(FT, 1) fsim_inv_rows_seq_kernel(FsimGroup g, const __grid_constant__ FftLen L, int wl, int sb,
                                                               int consts_mode, double *rowsums) {
    extern __shared__ __align__(16) float2 sm[];
    __shared__ double red[4][FT / 32];
    const int y = blockIdx.x, o = blockIdx.y, plane = blockIdx.z;
    const int w2 = g.w2;
    const float2 *src = g.T + (size_t(plane) * 16 + o * 4) * g.n + size_t(y) * w2;
    float2 *keep = sm;  // 4 x w2
    float2 *a = sm + 4 * w2, *b = a + size_t(sb) * wl;  // sb x wl each
    for (int s0 = 0; s0 < 4; s0 += sb) {
        batched_copy<float2>(
            threadIdx.x, sb * w2, FT,
            [&](int idx) {
                const int t = idx / w2, x = idx - t * w2;
                return src[size_t(s0 + t) * g.n + x];
            },
            [&](int idx, float2 v) {
                const int t = idx / w2, x = idx - t * w2;
                a[size_t(t) * wl + x] = v;
            });
        const float2 *res = iqm::fft_run(a, b, L, 1.f, sb, wl);
        for (int idx = threadIdx.x; idx < sb * w2; idx += FT) {
            const int t = idx / w2, x = idx - t * w2;
            keep[(s0 + t) * w2 + x] = res[size_t(t) * wl + x];
        }
        __syncthreads();
    }
    const float invN = 1.0f / float(g.n);
    if (!consts_mode) {
        const size_t off = (size_t(g.pair0 * 2 + plane) * 4 + o) * g.n + size_t(y) * w2;
        for (int x = threadIdx.x; x < w2; x += FT) {
            float2 v[4];
#pragma unroll
            for (int q = 0; q < 4; q++) v[q] = keep[q * w2 + x];
            float sA, en, e0;
            response_sums(v, invN, sA, en, e0);
            g.amp[off + x] = sA;
            g.energy[off + x] = en;
            g.eo0[off + x] = e0;
        }
        return;
    }
    const long lim = (long(g.n) + 1) / 2;
    const float fn = float(g.n);
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int x = threadIdx.x; x < w2; x += FT) {
        float re[4];
#pragma unroll
        for (int q = 0; q < 4; q++) re[q] = keep[q * w2 + x].x * invN;
        float q2 = 0.f, qx = 0.f;
#pragma unroll
        for (int q = 0; q < 4; q++) q2 += (re[q] * re[q]) * fn;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = i + 1; j < 4; j++) qx += re[i] * re[j] * fn;
        const long p = long(y) * w2 + x;
        if (p < lim) {
            acc[0] += q2;
            acc[1] += qx;
        }
        acc[2] += q2;
        acc[3] += qx;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        double v = acc[q];
        for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
        if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0.0;
        for (int i = 0; i < FT / 32; i++) t += red[threadIdx.x][i];
        rowsums[(size_t(o) * g.h2 + y) * 4 + threadIdx.x] = t;
    }
}

// ---------------------------------------------------------------------------------------------
// Mixed precision (IQM_MIXED, IQM_MIXED_FAST): the inverse passes on the tensor cores.  Each
// transform is a two-factor DFT computed with FP16 mma.sync tiles and FP32 accumulation
// (dft_mma.cuh); the spectrum is scaled by 1/N as the column pass loads it, so every FP16 operand
// and the FP16 intermediate planes between the passes stay in range, and the row pass produces the
// normalised responses directly.  Both kernels are persistent: each warp builds its transform's
// constant fragments once and the CTAs stride over (columns or rows, orientation, plane) items.

// Column pass: a work item is MCW adjacent columns of one (orientation, pair); warp c transforms
// column c of both images for the orientation's 4 scales.  The pair's packed spectrum is read once
// per item and separated into both images' spectra in a shared slab, each column stored as N1
// segments of N2 points padded to a stride of SEG (conflict-free loads by the engine's lane
// pattern); each scale's outputs are staged as FP16 rows of MCW columns and written to the
// intermediate planes as 16-byte row segments.
constexpr int MCW = 8;
template <class Dft>
struct MmaColGeom {
    static constexpr int H = Dft::N;                                      // column length
    static constexpr int SEG = Dft::N2 + ((4 - Dft::N2 % 16) + 16) % 16;  // N2 padded to 4 mod 16
    static constexpr int SLAB = Dft::N1 * SEG;                            // padded column, float2
    // staging row stride (half2): MCW columns; odd, so the 32 lanes' scattered output rows
    // k = g + 15 t (+ const) fall at most 2 to a bank (a multiple of 4 puts them 4 to a bank)
    static constexpr int SP = 13;
    static constexpr size_t tables = Dft::smem_bytes;
    static constexpr size_t slab_bytes = sizeof(float2) * 2 * MCW * SLAB;
    static constexpr int FLD = (H + 3) & ~3;  // per-warp filter column (floats), 16-byte aligned
    static constexpr size_t stage_bytes = sizeof(__half2) * 2 * H * SP;
    static constexpr size_t smem = tables + slab_bytes + stage_bytes + sizeof(float) * MCW * FLD;
    static_assert(MCW == 8 && tables % 16 == 0 && slab_bytes % 16 == 0, "16-byte aligned slab and staging");
};

template <class Dft>
// Single-product engines with shared tables fit 3 CTAs per SM without spills; the others 2.
__global__ void __launch_bounds__(32 * MCW, Dft::P == 1 && !Dft::kRegs ? 3 : 2)
    fsim_inv_cols_mma_kernel(FsimGroup g, const void *__restrict__ table, int items) {
    using Gm = MmaColGeom<Dft>;
    constexpr int H = Gm::H;
    extern __shared__ __align__(16) float2 sm[];
    float2 *Sl = sm + Gm::tables / sizeof(float2);                          // [img][column][SLAB]
    __half2 *stage = reinterpret_cast<__half2 *>(Sl + 2 * MCW * Gm::SLAB);  // [img][y][SP]
    const int warp = threadIdx.x >> 5;
    // this warp's column of the current filter, read once per scale for both images
    float *fcol = reinterpret_cast<float *>(reinterpret_cast<unsigned char *>(stage) + Gm::stage_bytes) + warp * Gm::FLD;
    Dft dft;
    dft.load(table, sm);  // complete at the item loop's first barrier
    const int ngroups = (g.w2 + MCW - 1) / MCW;
    const float hs = 0.5f / float(g.n);
    for (int item = blockIdx.x; item < items; item += gridDim.x) {
        const int cg = item % ngroups;
        const int o = (item / ngroups) & 3;
        const int pr = item / (ngroups * 4);  // chunk-local pair
        const int x0 = cg * MCW, nc = min(MCW, g.w2 - x0);
        const float2 *src = g.spec + size_t(g.pair0 + pr) * g.n;
        for (int idx = threadIdx.x; idx < MCW * H; idx += blockDim.x) {
            const int y = idx / MCW, c = idx - y * MCW;
            float2 v0 = make_float2(0.f, 0.f), v1 = v0;
            if (c < nc) {
                const int x = x0 + c;
                // Z = F(Y_img + i Y_ref): F(Y_img) = (Z(k) + conj Z(-k)) / 2, F(Y_ref) = (Z(k) - conj Z(-k)) / 2i
                const float2 z = src[size_t(y) * g.w2 + x];
                const float2 m = src[size_t(y ? H - y : 0) * g.w2 + (x ? g.w2 - x : 0)];
                v0 = make_float2(hs * (z.x + m.x), hs * (z.y - m.y));
                v1 = make_float2(hs * (z.y + m.y), hs * (m.x - z.x));
            }
            const int si = c * Gm::SLAB + (y / Dft::N2) * Gm::SEG + y % Dft::N2;
            Sl[si] = v0;
            Sl[MCW * Gm::SLAB + si] = v1;
        }
        __syncthreads();
#pragma unroll 1
        for (int s = 0; s < 4; s++) {
            if (warp < nc) {  // warp-uniform
                const float *Hz = g.filters + size_t(o * 4 + s) * g.n + size_t(x0 + warp) * H;
                for (int i = threadIdx.x & 31; i < H; i += 32) fcol[i] = __ldg(Hz + i);
                __syncwarp();
#pragma unroll 1
                for (int img = 0; img < 2; img++) {
                    const float2 *col = Sl + (img * MCW + warp) * Gm::SLAB;
                    __half2 *st = stage + img * H * Gm::SP + warp;
                    dft.run(
                        [&](int n1, int n2) {
                            const float h = fcol[Dft::N2 * n1 + n2];
                            const float2 v = col[n1 * Gm::SEG + n2];
                            return make_float2(h * v.x, h * v.y);
                        },
                        [&](int k, int, float2 v) { st[k * Gm::SP] = __floats2half2_rn(v.x, v.y); });
                }
            }
            __syncthreads();
            const size_t zoff = size_t(o * 4 + s) * g.n + size_t(x0);
            if (nc == MCW) {
                for (int idx = threadIdx.x; idx < 2 * H * 2; idx += blockDim.x) {
                    const int q = idx & 1, r = idx >> 1;  // r = img * H + y
                    const int img = r / H, y = r - img * H;
                    const unsigned *row = reinterpret_cast<const unsigned *>(stage + r * Gm::SP + 4 * q);
                    const uint4 v = make_uint4(row[0], row[1], row[2], row[3]);
                    *reinterpret_cast<uint4 *>(g.Th + size_t(2 * pr + img) * 16 * g.n + zoff + size_t(y) * g.w2 + 4 * q) = v;
                }
            } else {
                for (int idx = threadIdx.x; idx < 2 * H * MCW; idx += blockDim.x) {
                    const int c = idx % MCW, r = idx / MCW;
                    const int img = r / H, y = r - img * H;
                    if (c < nc) g.Th[size_t(2 * pr + img) * 16 * g.n + zoff + size_t(y) * g.w2 + c] = stage[r * Gm::SP + c];
                }
            }
            __syncthreads();  // staging rows read before the next scale overwrites them
        }
    }
}

// The 32 bits of an FP16 pair, to go into an MMA operand unchanged.
__device__ __forceinline__ unsigned h2_word(__half2 h) { return *reinterpret_cast<unsigned *>(&h); }

// Row pass: a work item is one row of one (orientation, plane), taken by one warp on its own: it
// transforms the row for the 4 scales, reading its FP16 inputs straight from the intermediate
// planes, parks the first 3 scales' outputs in its own shared slots and keeps the last in
// registers, then forms the response sums of its outputs (as fsim_inv_rows_kernel does) and
// stores them; no barrier after the tables are loaded.
constexpr int MRW = 8;  // warps per CTA of the row pass
template <class Dft>
struct MmaRowGeom {
    static constexpr int W = Dft::N;
    static constexpr int SLOTS = 2 * Dft::NTC;  // output slots per lane
    static constexpr size_t tables = Dft::smem_bytes;
    static constexpr size_t smem = tables + sizeof(float2) * MRW * 3 * SLOTS * 32;
};

template <class Dft>
__global__ void __launch_bounds__(32 * MRW, Dft::P == 1 ? 2 : 1)
    fsim_inv_rows_mma_kernel(FsimGroup g, const void *__restrict__ table, int items) {
    using Gm = MmaRowGeom<Dft>;
    constexpr int W = Gm::W, SL = Gm::SLOTS;
    extern __shared__ __align__(16) float2 sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float2 *keep = sm + Gm::tables / sizeof(float2) + size_t(warp) * 3 * SL * 32;  // [scale][slot][lane]
    Dft dft;
    dft.load(table, sm);
    __syncthreads();
    for (int item = blockIdx.x * MRW + warp; item < items; item += gridDim.x * MRW) {  // warp-uniform
        const int y = item % g.h2;
        const int o = (item / g.h2) & 3;
        const int plane = item / (g.h2 * 4);  // chunk-local pair*2 + img
        float2 last[SL];
#pragma unroll 1
        for (int s = 0; s < 4; s++) {
            const __half2 *src = g.Th + (size_t(plane) * 16 + o * 4 + s) * g.n + size_t(y) * W;
            dft.run([&](int n1, int n2) { return h2_word(src[Dft::N2 * n1 + n2]); },
                    [&](int, int slot, float2 v) {
                        if (s < 3)
                            keep[(s * SL + slot) * 32 + lane] = v;
                        else
                            last[slot] = v;
                    });
        }
        const size_t row = (size_t(g.pair0 * 2 + plane) * 4 + o) * g.n + size_t(y) * W;
#pragma unroll
        for (int slot = 0; slot < SL; slot++) {
            const int k1 = Dft::slot_k1(slot), k2 = Dft::slot_k2(slot);
            if (k1 >= Dft::N1 || k2 >= Dft::N2) continue;
            const int x = k1 + Dft::N1 * k2;
            const float2 v[4] = {keep[slot * 32 + lane], keep[(SL + slot) * 32 + lane], keep[(2 * SL + slot) * 32 + lane],
                                 last[slot]};
            float sA, en, e0;
            response_sums(v, 1.0f, sA, en, e0);  // already normalised
            g.amp[row + x] = sA;
            g.energy[row + x] = en;
            g.eo0[row + x] = e0;
        }
    }
}

// Builds an engine's constant table (one warp).
template <class Dft>
__global__ void mma_table_kernel(void *table) {
    Dft::build(table, 1.f);
}

// Tensor-core transform engines of the mixed forms: 270 = 15 x 18 (columns), 480 = 16 x 30 (rows).
// Single products keep the column engine's stage-C matrix and twiddles in registers (measured 5%
// faster than the shared table at 1080p); split products keep them in shared memory (registers
// would spill).
template <int SPLIT>
using MmaCol270 = iqm::MmaDft<15, 18, SPLIT, SPLIT == 1>;
template <int SPLIT>
using MmaRow480 = iqm::MmaDft<16, 30, SPLIT>;

// sum the per-row constants in row order -> an2[mode][o], aiaj[mode][o]
__global__ void fsim_consts_reduce_kernel(const double *rowsums, int h2, double *consts) {
    const int o = threadIdx.x;  // 4 threads
    if (o >= 4) return;
    double t[4] = {0.0, 0.0, 0.0, 0.0};
    for (int y = 0; y < h2; y++)
        for (int q = 0; q < 4; q++) t[q] += rowsums[(size_t(o) * h2 + y) * 4 + q];
    consts[4 + 0 * 4 + o] = t[0];   // an2 [ref]
    consts[12 + 0 * 4 + o] = t[1];  // aiaj[ref]
    consts[4 + 1 * 4 + o] = t[2];   // an2 [full]
    consts[12 + 1 * 4 + o] = t[3];  // aiaj[full]
}

// ---------------------------------------------------------------------------------------------
// noise power and threshold -- src/gpu/fsim/steps/fsim_noise_power.cpp:193-205 (upper median of a
// full sort, mean = -median/ln 0.5, divided by EM_n(o)) and shaders/fsim/fsim_phase_congruency.glsl:
// 42-53 (estimated noise energy, tau, T = (mu + k sigma)/1.7 with k = 2); evaluated in FP64.
constexpr int NOISE_STAGE = 7168;  // 28 KB: 16 KB of histogram beside it stays under 48 KB
// two CTAs per SM: 8 planes x 32 pairs run in one wave on 148 SMs
__global__ void __launch_bounds__(1024, 2) fsim_noise_kernel(FsimGroup g) {
    __shared__ unsigned hist[iqm::SELECT_BINS];
    __shared__ unsigned stage[NOISE_STAGE];  // the median's first-digit bucket, when it fits
    const int q = blockIdx.x;   // img*4 + o
    const int pi = blockIdx.y;
    const int o = q & 3;
    const float *v = g.eo0 + (size_t(pi) * 8 + q) * g.n;
    const float med = iqm::block_select_kth(v, g.n, g.n / 2, hist, stage, NOISE_STAGE);
    if (threadIdx.x == 0) {
        const double mean = -double(med) / log(0.5);
        const double np = mean / g.consts[o];
        const double an2 = g.consts[4 + g.energy_mode * 4 + o];
        const double aiaj = g.consts[12 + g.energy_mode * 4 + o];
        const double e2 = 2.0 * np * an2 + 4.0 * np * aiaj;
        const double tau = sqrt(e2 / 2.0);
        const double mu = tau * sqrt(GLSL_PI / 2.0);
        const double sig = sqrt((2.0 - GLSL_PI / 2.0) * (tau * tau));
        g.thr[size_t(pi) * 8 + q] = float((mu + 2.0 * sig) / 1.7);
    }
}

// ---------------------------------------------------------------------------------------------
// phase congruency (fsim_phase_congruency.glsl:39-64), gradient (fsim_gradientmap.glsl:16-57),
// similarities (fsim_final_multiply.glsl:18-58; T1 0.85, T2 160, T3 = T4 200, lambda 0.03) and the
// pooled sums (fsim_final_multiply.cpp:294-300), FP64 accumulation.
__device__ __forceinline__ float grad_at(const float *Y, int x, int y, int w2, int h2) {
    const float vert[9] = {3.f, 0.f, -3.f, 10.f, 0.f, -10.f, 3.f, 0.f, -3.f};
    const float hor[9] = {3.f, 10.f, 3.f, 0.f, 0.f, 0.f, -3.f, -10.f, -3.f};
    float vs = 0.f, hs = 0.f;
#pragma unroll
    for (int j = -1; j < 2; j++)
#pragma unroll
        for (int k = -1; k < 2; k++) {
            const int px = x + j, py = y + k;
            if (px >= 0 && px < w2 && py >= 0 && py < h2) {
                const float v = Y[py * w2 + px];
                const int idx = (j + 1) + (k + 1) * 3;
                vs += v * vert[idx];
                hs += v * hor[idx];
            }
        }
    const float a = vs / 16.0f, b = hs / 16.0f;
    return iqm::sqrt_nonneg(a * a + b * b);
}

// Similarity terms of one pixel from the two images' phase congruency, gradient magnitude and
// chroma (fsim_final_multiply.glsl:18-58).
__device__ __forceinline__ void similarity_terms(float pc1, float pc2, float g1, float g2, float i1, float i2, float q1,
                                                 float q2, double &s_pcm, double &s_sim, double &s_simc) {
    const float pcm = fmaxf(pc1, pc2);
    // denominators >= 0.85: SFU reciprocals; |SI SQ|^0.03 as exp2(0.03 log2 |SI SQ|) (0 for 0)
    const float pcsim = (2.0f * pc1 * pc2 + 0.85f) * iqm::rcp_approx(pc1 * pc1 + pc2 * pc2 + 0.85f);
    const float gsim = (2.0f * g1 * g2 + 160.0f) * iqm::rcp_approx(g1 * g1 + g2 * g2 + 160.0f);
    const float isim = (2.0f * i1 * i2 + 200.0f) * iqm::rcp_approx(i1 * i1 + i2 * i2 + 200.0f);
    const float qsim = (2.0f * q1 * q2 + 200.0f) * iqm::rcp_approx(q1 * q1 + q2 * q2 + 200.0f);
    const float sim = gsim * pcsim * pcm;
    const float simc = gsim * pcsim * iqm::ex2_approx(0.03f * iqm::lg2_approx(fabsf(isim * qsim))) * pcm;
    s_pcm += pcm;
    s_sim += sim;
    s_simc += simc;
}

// PX pixels per thread: 1, or 4 consecutive pixels of one row read with 16-byte loads (w2 a
// multiple of 4, so every plane starts 16-byte aligned and no quad crosses a row).
template <int PX>
__global__ void __launch_bounds__(FT) fsim_final_kernel(FsimGroup g) {
    __shared__ double red[3][FT / 32];
    __shared__ int is_last;
    const int pi = blockIdx.y;
    const int p = (blockIdx.x * FT + threadIdx.x) * PX;
    const int n = g.n;
    double s_pcm = 0.0, s_sim = 0.0, s_simc = 0.0;
    if constexpr (PX == 4) {
        if (p < n) {
            const int w2 = g.w2, h2 = g.h2;
            const int x0 = p % w2, y = p / w2;
            float pc[2][4], gm[2][4], iv[2][4], qv[2][4];
#pragma unroll
            for (int img = 0; img < 2; img++) {
                float et[4] = {0.f, 0.f, 0.f, 0.f}, at[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                for (int o = 0; o < 4; o++) {
                    const size_t plane = (size_t(pi) * 8 + img * 4 + o) * n;
                    const float4 e = __ldcs(reinterpret_cast<const float4 *>(g.energy + plane + p));
                    const float4 a = __ldcs(reinterpret_cast<const float4 *>(g.amp + plane + p));
                    const float t = g.thr[size_t(pi) * 8 + img * 4 + o];
                    et[0] += fmaxf(e.x - t, 0.f);
                    et[1] += fmaxf(e.y - t, 0.f);
                    et[2] += fmaxf(e.z - t, 0.f);
                    et[3] += fmaxf(e.w - t, 0.f);
                    at[0] += a.x;
                    at[1] += a.y;
                    at[2] += a.z;
                    at[3] += a.w;
                }
#pragma unroll
                for (int j = 0; j < 4; j++) pc[img][j] = et[j] / at[j];
                const float *yiq = g.yiq + size_t(pi * 2 + img) * 3 * n;
                const float4 i4 = *reinterpret_cast<const float4 *>(yiq + p);
                const float4 q4 = *reinterpret_cast<const float4 *>(yiq + n + p);
                iv[img][0] = i4.x, iv[img][1] = i4.y, iv[img][2] = i4.z, iv[img][3] = i4.w;
                qv[img][0] = q4.x, qv[img][1] = q4.y, qv[img][2] = q4.z, qv[img][3] = q4.w;
                // 3 x 6 luma window around the quad, zero outside the plane (grad_at's skipped samples)
                const float *Y = yiq + 2 * n;
                float win[3][6];
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    const int py = y + r - 1;
                    if (py >= 0 && py < h2) {
                        const float *row = Y + size_t(py) * w2;
                        const float4 c = *reinterpret_cast<const float4 *>(row + x0);
                        win[r][0] = x0 > 0 ? row[x0 - 1] : 0.f;
                        win[r][1] = c.x, win[r][2] = c.y, win[r][3] = c.z, win[r][4] = c.w;
                        win[r][5] = x0 + 4 < w2 ? row[x0 + 4] : 0.f;
                    } else {
#pragma unroll
                        for (int c = 0; c < 6; c++) win[r][c] = 0.f;
                    }
                }
                const float vert[9] = {3.f, 0.f, -3.f, 10.f, 0.f, -10.f, 3.f, 0.f, -3.f};
                const float hor[9] = {3.f, 10.f, 3.f, 0.f, 0.f, 0.f, -3.f, -10.f, -3.f};
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    float vs = 0.f, hs = 0.f;
#pragma unroll
                    for (int dj = -1; dj < 2; dj++)
#pragma unroll
                        for (int dk = -1; dk < 2; dk++) {
                            const float v = win[dk + 1][q + 1 + dj];
                            const int idx = (dj + 1) + (dk + 1) * 3;
                            vs += v * vert[idx];
                            hs += v * hor[idx];
                        }
                    const float a = vs / 16.0f, b = hs / 16.0f;
                    gm[img][q] = iqm::sqrt_nonneg(a * a + b * b);
                }
            }
#pragma unroll
            for (int q = 0; q < 4; q++)
                similarity_terms(pc[0][q], pc[1][q], gm[0][q], gm[1][q], iv[0][q], iv[1][q], qv[0][q], qv[1][q], s_pcm,
                                 s_sim, s_simc);
        }
    } else if (p < n) {
        float pc[2];
#pragma unroll
        for (int img = 0; img < 2; img++) {
            float et = 0.f, at = 0.f;
#pragma unroll
            for (int o = 0; o < 4; o++) {
                const size_t plane = (size_t(pi) * 8 + img * 4 + o) * n;
                const float e = g.energy[plane + p] - g.thr[size_t(pi) * 8 + img * 4 + o];
                et += fmaxf(e, 0.f);
                at += g.amp[plane + p];
            }
            pc[img] = et / at;
        }
        const int x = p % g.w2, y = p / g.w2;
        const float *yiq1 = g.yiq + size_t(pi * 2 + 0) * 3 * n;
        const float *yiq2 = g.yiq + size_t(pi * 2 + 1) * 3 * n;
        const float g1 = grad_at(yiq1 + 2 * n, x, y, g.w2, g.h2);
        const float g2 = grad_at(yiq2 + 2 * n, x, y, g.w2, g.h2);
        similarity_terms(pc[0], pc[1], g1, g2, yiq1[p], yiq2[p], yiq1[n + p], yiq2[n + p], s_pcm, s_sim, s_simc);
    }
    double v[3] = {s_pcm, s_sim, s_simc};
#pragma unroll
    for (int q = 0; q < 3; q++) {
        for (int d = 16; d > 0; d >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], d);
        if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v[q];
    }
    __syncthreads();
    double *part = g.partials + (size_t(pi) * g.tiles + blockIdx.x) * 3;
    if (threadIdx.x < 3) {
        double t = 0.0;
        for (int i = 0; i < FT / 32; i++) t += red[threadIdx.x][i];
        part[threadIdx.x] = t;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(&g.counters[pi], 1u);
        is_last = prev == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    {
        double t[3] = {0.0, 0.0, 0.0};
        const double *pp = g.partials + size_t(pi) * g.tiles * 3;
        for (int i = threadIdx.x; i < int(gridDim.x); i += FT)
#pragma unroll
            for (int q = 0; q < 3; q++) t[q] += __ldcg(pp + size_t(i) * 3 + q);
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 3; q++) {
            for (int d = 16; d > 0; d >>= 1) t[q] += __shfl_down_sync(0xffffffffu, t[q], d);
            if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = t[q];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot[3] = {0.0, 0.0, 0.0};
        for (int i = 0; i < FT / 32; i++)
            for (int q = 0; q < 3; q++) tot[q] += red[q][i];
        const int out = g.pairs[pi].out;
        g.scores[2 * out] = tot[1] / tot[0];
        g.scores[2 * out + 1] = tot[2] / tot[0];
        g.counters[pi] = 0u;
    }
}

// ---------------------------------------------------------------------------------------------
// host orchestration

int downscale_factor(int w, int h) {  // src/gpu/fsim/fsim.cpp:165-168
    const int smaller = std::min(w, h);
    return std::max(1, int(std::round(smaller / 256.0)));
}

void plane_size(int w, int h, int F, int &w2, int &h2) {  // src/gpu/fsim/fsim.cpp:91-92
    w2 = int(std::round(float(w) / float(F)));
    h2 = int(std::round(float(h) / float(F)));
}

constexpr size_t SMEM_CAP = 200 * 1024;
constexpr int kFsimStreams = 8;  // plane-size groups in flight at once
constexpr bool kOverlapChunks = true;  // rotate inverse-pass chunks over several streams
// Streams (and L2-sized buffers) the chunks rotate over: two fill each other's partial waves; three
// measured 2% slower (the third chunk's planes crowd the L2).
constexpr int kChunkStreams = 2;
static_assert(kChunkStreams >= 1 && kChunkStreams <= 8, "chunk streams");

// Raises a kernel's dynamic shared-memory limit on the current device to at least `bytes` (never
// lowers it: launches already enqueued or captured for other plane sizes keep their sizes valid).
void set_smem(const void *fn, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, size_t> current;  // kernel attributes are per device
    int dev = 0;
    IQM_CHECK_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_pair(dev, fn);
    auto it = current.find(key);
    if (it == current.end()) {
        // transform CTAs are shared-memory bound: ask for the largest shared-memory carveout so
        // as many CTAs fit per SM as registers allow
        IQM_CHECK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        it = current.emplace(key, 0).first;
    }
    if (bytes <= 48 * 1024 || bytes <= it->second) return;
    IQM_CHECK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    it->second = bytes;
}

// Launch shapes of the transform kernels for one plane size.
struct Shapes {
    int wl_row, wl_col;   // work lengths (n, or Bluestein m)
    int lw_rows;          // log2 warps per CTA, forward rows (NB rows per warp)
    int lw_fcols;         // log2 warps per CTA, forward columns (NB columns per warp)
    int lw_icols;         // log2 warps per CTA, inverse columns
    int rr;               // rows per CTA in the inverse row pass (0: sequential kernel)
    int icols_cb;         // columns per CTA of the CTA-wide inverse column pass (0: warp kernel)
    int seq_sb;           // scales per engine call of the sequential row kernel
    int row_eng, col_eng; // transform engine of the row / column length (engine_id)
    size_t sm_rows, sm_fcols, sm_icols, sm_irows, sm_icols_seq;
};

// Compiled transform engine serving a length: 1 (270) or 2 (480) when the length's own plan is
// exactly the compiled radix sequence, else 0 (the runtime-planned engine).
int engine_id(const iqm::FftLen &L) {
    auto is = [&](int n, std::initializer_list<int> rs) {
        if (L.bluestein || L.n != n || L.nst != int(rs.size())) return false;
        int i = 0;
        for (int r : rs)
            if (L.radix[i++] != r) return false;
        return true;
    };
    if (is(270, {9, 3, 10})) return 1;
    if (is(480, {15, 8, 4})) return 2;
    return 0;
}

// Work buffers per warp of engine `id` (matches engine_bufs of the types with_engine selects).
int engine_buffers(int id) { return id == 2 ? 1 : 2; }
static_assert(engine_bufs<Engine270>::value == 2 && engine_bufs<Engine480>::value == 1 &&
                  engine_bufs<GenericEngine>::value == 2,
              "engine_buffers() must match the engines' work buffers");

template <class F>
void with_engine(int id, F &&f) {
    switch (id) {
        case 1: f(Engine270{}); break;
        case 2: f(Engine480{}); break;
        default: f(GenericEngine{}); break;
    }
}

// Warps of a kernel resident per SM at this block size and dynamic shared memory (raises the
// kernel's shared-memory limit first, as a launch would).  Memoised per device: plane shapes are
// chosen on every enqueue.
int resident_warps(const void *fn, int threads, size_t smem) {
    static std::mutex mu;
    static std::map<std::tuple<int, const void *, int, size_t>, int> known;
    int dev = 0;
    IQM_CHECK_CUDA(cudaGetDevice(&dev));
    const auto key = std::make_tuple(dev, fn, threads, smem);
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = known.find(key);
        if (it != known.end()) return it->second;
    }
    set_smem(fn, smem);
    int blocks = 0;
    IQM_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, threads, smem));
    const int warps = blocks * threads / 32;
    std::lock_guard<std::mutex> lock(mu);
    known[key] = warps;
    return warps;
}

int lw_fit(size_t fixed, size_t per_warp) {
    int lw = 3;  // up to 8 warps
    while (lw > 0 && fixed + (size_t(1) << lw) * per_warp > 160 * 1024) lw--;
    return lw;
}

Shapes shapes_for(const iqm::FsimPlan &P, const iqm::FsimTune &tune = iqm::FsimTune{}) {
    Shapes s{};
    const size_t f2 = sizeof(float2);
    s.wl_row = iqm::fft_work_len(P.row);
    s.wl_col = iqm::fft_work_len(P.col);
    s.row_eng = engine_id(P.row);
    s.col_eng = engine_id(P.col);
    const size_t twr = size_t((iqm::stage_twiddle_len(P.row) + 1) & ~1) * f2;
    const size_t twc = size_t((iqm::stage_twiddle_len(P.col) + 1) & ~1) * f2;
    const size_t warp_row = engine_buffers(s.row_eng) * NB * size_t(s.wl_row) * f2;
    const size_t warp_col = engine_buffers(s.col_eng) * NB * size_t(s.wl_col) * f2;
    s.lw_rows = lw_fit(twr, warp_row);
    s.sm_rows = twr + (size_t(1) << s.lw_rows) * warp_row;
    s.lw_fcols = lw_fit(twc, warp_col);
    s.sm_fcols = twc + (size_t(1) << s.lw_fcols) * warp_col;
    s.lw_icols = lw_fit(twc, warp_col + NB * size_t(P.h2) * f2);
    if (tune.icols_lw >= 0) s.lw_icols = std::min(s.lw_icols, tune.icols_lw);
    s.sm_icols = twc + (size_t(1) << s.lw_icols) * (warp_col + NB * size_t(P.h2) * f2);
    // Runtime-planned columns: the CTA-wide column kernel (cb columns per CTA, the most warps resident
    // per SM) when it keeps at least twice as many warps resident as the warp kernel, whose per-warp
    // work buffers grow with the length.
    if (s.col_eng == 0) {
        const int w_warp = resident_warps((const void *)fsim_inv_cols_kernel<GenericEngine>, 32 << s.lw_icols, s.sm_icols);
        int best = 0;
        for (int cb : {4, 2, 1}) {
            const size_t sm = size_t(cb) * (size_t(P.h2) + 2 * size_t(s.wl_col)) * f2;
            if (sm > SMEM_CAP) continue;
            const int w = resident_warps((const void *)fsim_inv_cols_seq_kernel, FT, sm);
            if (w >= 2 * w_warp && w > best) {
                best = w;
                s.icols_cb = cb;
                s.sm_icols_seq = sm;
            }
        }
    }
    const size_t per_row = (4 / NB) * warp_row;  // 4/NB warps per row (four scales)
    if (twr + 2 * per_row <= 120 * 1024) {
        s.rr = 2;
    } else if (twr + per_row <= SMEM_CAP) {
        s.rr = 1;
    } else {
        s.rr = 0;
    }
    if (s.rr && tune.rows_per_cta >= 1 && tune.rows_per_cta < s.rr) s.rr = tune.rows_per_cta;
    // The sequential row kernel transforms seq_sb scales per engine call: the choice with the most
    // transforms in flight per SM, and on a tie the one with more CTAs per SM.
    s.seq_sb = 1;
    if (!s.rr) {
        int best = -1;
        for (int sb : {1, 2, 4}) {
            const size_t sm = (4 * size_t(P.w2) + 2 * size_t(sb) * s.wl_row) * f2;
            if (sm > SMEM_CAP) continue;
            const int inflight = resident_warps((const void *)fsim_inv_rows_seq_kernel, FT, sm) / (FT / 32) * sb;
            if (inflight > best) {
                best = inflight;
                s.seq_sb = sb;
            }
        }
    }
    s.sm_irows = s.rr ? twr + s.rr * per_row : (4 * size_t(P.w2) + 2 * size_t(s.seq_sb) * s.wl_row) * f2;
    IQM_REQUIRE(s.sm_rows <= SMEM_CAP && s.sm_fcols <= SMEM_CAP && s.sm_icols <= SMEM_CAP && s.sm_irows <= SMEM_CAP,
                "FSIM plane too large for the shared-memory FFT");
    return s;
}

void configure_kernels(const Shapes &s) {
    with_engine(s.row_eng, [&](auto e) {
        using E = decltype(e);
        set_smem((const void *)fsim_fwd_rows_kernel<E>, s.sm_rows);
        if (s.rr) set_smem((const void *)fsim_inv_rows_kernel<E>, s.sm_irows);
    });
    with_engine(s.col_eng, [&](auto e) {
        using E = decltype(e);
        set_smem((const void *)fsim_fwd_cols_kernel<E>, s.sm_fcols);
        set_smem((const void *)fsim_inv_cols_kernel<E>, s.sm_icols);
    });
    if (!s.rr) {
        set_smem((const void *)fsim_inv_rows_seq_kernel, s.sm_irows);
    }
    if (s.icols_cb) set_smem((const void *)fsim_inv_cols_seq_kernel, s.sm_icols_seq);
}

void launch_inv_rows(const FsimGroup &g, const iqm::FsimPlan &P, const Shapes &s, int planes, int consts_mode,
                     double *rowsums, cudaStream_t st) {
    if (s.rr && !(consts_mode && s.rr != 1)) {
        with_engine(s.row_eng, [&](auto e) {
            fsim_inv_rows_kernel<decltype(e)>
                <<<dim3(iqm::ceil_div(P.h2, s.rr), 4, planes), 32 * (4 / NB) * s.rr, s.sm_irows, st>>>(
                    g, P.row, s.wl_row, s.rr, consts_mode, rowsums);
        });
    } else if (s.rr) {  // consts mode runs one row per CTA
        const size_t twr = size_t((iqm::stage_twiddle_len(P.row) + 1) & ~1) * sizeof(float2);
        with_engine(s.row_eng, [&](auto e) {
            fsim_inv_rows_kernel<decltype(e)><<<dim3(P.h2, 4, planes), 32 * (4 / NB), twr + (s.sm_irows - twr) / s.rr, st>>>(
                g, P.row, s.wl_row, 1, 1, rowsums);
        });
    } else {
        fsim_inv_rows_seq_kernel<<<dim3(P.h2, 4, planes), FT, s.sm_irows, st>>>(g, P.row, s.wl_row, s.seq_sb,
                                                                                 consts_mode, rowsums);
    }
}

void launch_inv_cols(const FsimGroup &g, const iqm::FsimPlan &P, const Shapes &s, int planes, int consts_mode,
                     cudaStream_t st) {
    if (s.icols_cb && !consts_mode) {
        fsim_inv_cols_seq_kernel<<<dim3(iqm::ceil_div(P.w2, s.icols_cb), 4, planes), FT, s.sm_icols_seq, st>>>(
            g, P.col, s.wl_col, s.icols_cb);
        return;
    }
    const int nw = 1 << s.lw_icols;
    with_engine(s.col_eng, [&](auto e) {
        fsim_inv_cols_kernel<decltype(e)><<<dim3(iqm::ceil_div(P.w2, NB * nw), 4, planes), 32 * nw, s.sm_icols, st>>>(
            g, P.col, s.wl_col, s.lw_icols, consts_mode);
    });
}

iqm::FsimPlan *get_plan(iqm_ctx *ctx, int w2, int h2) {
    auto key = std::make_pair(w2, h2);
    auto it = ctx->fsim_plans.find(key);
    if (it != ctx->fsim_plans.end()) return it->second;
    auto *P = new iqm::FsimPlan();
    P->w2 = w2;
    P->h2 = h2;
    P->n = w2 * h2;
    const int n = P->n;
    void *tmp = nullptr;
    try {
        P->row = iqm::fft_len(ctx, w2);
        P->col = iqm::fft_len(ctx, h2);
        IQM_CHECK_CUDA(cudaMalloc(&P->filters, sizeof(float) * 16 * size_t(n)));
        IQM_CHECK_CUDA(cudaMalloc(&P->consts, sizeof(double) * 20));
        const Shapes s = shapes_for(*P);
        configure_kernels(s);
        cudaStream_t st = ctx->stream;
        fsim_filters_kernel<<<iqm::ceil_div(n, FT), FT, 0, st>>>(P->filters, w2, h2);
        IQM_CHECK_CUDA(cudaGetLastError());
        fsim_em_kernel<<<4, FT, 0, st>>>(P->filters, n, P->consts);
        IQM_CHECK_CUDA(cudaGetLastError());
        // transforms of the filters themselves
        const size_t tbytes = sizeof(float2) * 16 * size_t(n);
        const size_t rbytes = sizeof(double) * 4 * 4 * size_t(h2);
        IQM_CHECK_CUDA(cudaMalloc(&tmp, tbytes + rbytes));
        FsimGroup g{};
        g.G = 1;
        g.w2 = w2;
        g.h2 = h2;
        g.n = n;
        g.T = static_cast<float2 *>(tmp);
        g.filters = P->filters;
        double *rowsums = reinterpret_cast<double *>(static_cast<uint8_t *>(tmp) + tbytes);
        launch_inv_cols(g, *P, s, 1, 1, st);
        IQM_CHECK_CUDA(cudaGetLastError());
        launch_inv_rows(g, *P, s, 1, 1, rowsums, st);
        IQM_CHECK_CUDA(cudaGetLastError());
        fsim_consts_reduce_kernel<<<1, 32, 0, st>>>(rowsums, h2, P->consts);
        IQM_CHECK_CUDA(cudaGetLastError());
        double host[20];
        IQM_CHECK_CUDA(cudaMemcpyAsync(host, P->consts, sizeof(host), cudaMemcpyDeviceToHost, st));
        IQM_CHECK_CUDA(cudaStreamSynchronize(st));
        cudaFree(tmp);
        tmp = nullptr;
        for (int o = 0; o < 4; o++) {
            P->em[o] = host[o];
            for (int m = 0; m < 2; m++) {
                P->an2[m][o] = host[4 + m * 4 + o];
                P->aiaj[m][o] = host[12 + m * 4 + o];
            }
        }
    } catch (...) {
        if (tmp) cudaFree(tmp);
        delete P;
        throw;
    }
    ctx->fsim_plans[key] = P;
    return P;
}

struct Layout {
    size_t yiq, spec, T, planes, thr, partials, counters, total;
};

// G pairs of the group; chunk pairs' worth of inverse-pass intermediates.
// nbuf: inverse-pass intermediate buffers (2 when consecutive chunks alternate between two streams).
// tbytes: bytes per element of the intermediate planes (8: FP32 complex, 4: FP16 complex).
Layout layout_for(int G, int chunk, int n, int tiles, int nbuf = 1, size_t tbytes = sizeof(float2)) {
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    Layout L{};
    size_t off = 0;
    L.yiq = off; off += al(sizeof(float) * size_t(G) * 6 * n);
    L.spec = off; off += al(sizeof(float2) * size_t(G) * n);
    L.T = off; off += al(tbytes * size_t(nbuf) * chunk * 32 * n);
    L.planes = off; off += al(sizeof(float) * size_t(G) * 24 * n);
    L.thr = off; off += al(sizeof(float) * size_t(G) * 8);
    L.partials = off; off += al(sizeof(double) * size_t(G) * tiles * 3);
    L.counters = off; off += al(sizeof(unsigned) * size_t(G));
    L.total = off;
    return L;
}

// Inverse-pass chunk: the 32 intermediate planes of `chunk` pairs stay within an L2 budget
// (80 MB unless tuned).
int chunk_pairs(const iqm::FsimTune &t, int G, int n, size_t tbytes = sizeof(float2)) {
    const size_t budget = size_t(t.chunk_mb > 0 ? t.chunk_mb : 80) << 20;
    return std::max(1, std::min(G, int(budget / (tbytes * 32 * size_t(n)))));
}

// Tensor-core transform engines of the mixed forms exist for 480 x 270 planes (1080p and 4K pairs
// downscale to them); other plane sizes run the FP32 transforms in the mixed forms too.
bool mma_plane(int w2, int h2) { return w2 == 480 && h2 == 270; }

// CTAs of a persistent kernel: the items, or as many CTAs as fit on the device at once.
int persistent_grid(const void *fn, int threads, size_t smem, int items) {
    int dev = 0, sms = 0, per_sm = 0;
    IQM_CHECK_CUDA(cudaGetDevice(&dev));
    IQM_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    set_smem(fn, smem);
    IQM_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
    return std::max(1, std::min(items, sms * std::max(1, per_sm)));
}

// Offsets of the four engines' constant tables in FsimPlan::mma_tables.
struct MmaTableLayout {
    size_t col1, col3, row1, row3, total;
};
MmaTableLayout mma_table_layout() {
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    MmaTableLayout L{};
    L.col1 = 0;
    L.col3 = L.col1 + al(MmaCol270<1>::table_bytes);
    L.row1 = L.col3 + al(MmaCol270<3>::table_bytes);
    L.row3 = L.row1 + al(MmaRow480<1>::table_bytes);
    L.total = L.row3 + al(MmaRow480<3>::table_bytes);
    return L;
}

// pairs: pairs in the chunk (each item of the column pass covers both images of a pair).
template <int SPLIT>
void launch_inv_mma(const FsimGroup &g, const iqm::FsimPlan &P, int pairs, cudaStream_t st, iqm_ctx *ctx) {
    using C = MmaCol270<SPLIT>;
    using R = MmaRow480<SPLIT>;
    const MmaTableLayout TL = mma_table_layout();
    const uint8_t *tables = static_cast<const uint8_t *>(P.mma_tables);
    const int citems = int(iqm::ceil_div(g.w2, MCW)) * 4 * pairs;
    const size_t csm = MmaColGeom<C>::smem;
    const int cgrid = persistent_grid((const void *)fsim_inv_cols_mma_kernel<C>, 32 * MCW, csm, citems);
    fsim_inv_cols_mma_kernel<C><<<cgrid, 32 * MCW, csm, st>>>(g, tables + (SPLIT == 1 ? TL.col1 : TL.col3), citems);
    iqm::check_launch(ctx, "fsim_inv_cols_mma_kernel");
    const int ritems = g.h2 * 4 * 2 * pairs;
    const size_t rsm = MmaRowGeom<R>::smem;
    const int rgrid = persistent_grid((const void *)fsim_inv_rows_mma_kernel<R>, 32 * MRW, rsm,
                                      int(iqm::ceil_div(ritems, MRW)));
    fsim_inv_rows_mma_kernel<R><<<rgrid, 32 * MRW, rsm, st>>>(g, tables + (SPLIT == 1 ? TL.row1 : TL.row3), ritems);
    iqm::check_launch(ctx, "fsim_inv_rows_mma_kernel");
}

// The tensor-core engines' constant tables of a 480 x 270 plan, built once on the context stream.
void ensure_mma_tables(iqm_ctx *ctx, iqm::FsimPlan *P) {
    if (P->mma_tables) return;
    const MmaTableLayout TL = mma_table_layout();
    IQM_CHECK_CUDA(cudaMalloc(&P->mma_tables, TL.total));
    uint8_t *t = static_cast<uint8_t *>(P->mma_tables);
    mma_table_kernel<MmaCol270<1>><<<1, 32, 0, ctx->stream>>>(t + TL.col1);
    mma_table_kernel<MmaCol270<3>><<<1, 32, 0, ctx->stream>>>(t + TL.col3);
    mma_table_kernel<MmaRow480<1>><<<1, 32, 0, ctx->stream>>>(t + TL.row1);
    mma_table_kernel<MmaRow480<3>><<<1, 32, 0, ctx->stream>>>(t + TL.row3);
    IQM_CHECK_CUDA(cudaGetLastError());
}

void launch_ingest(const FsimGroup &g, int F_uniform, int tiles, cudaStream_t st) {
    const dim3 grid(tiles, g.G);
    switch (F_uniform) {
        case 1: fsim_ingest_kernel<1><<<grid, FT, 0, st>>>(g); break;
        case 2: fsim_ingest_kernel<2><<<grid, FT, 0, st>>>(g); break;
        case 4: fsim_ingest_kernel<4><<<grid, FT, 0, st>>>(g); break;
        case 8: fsim_ingest_kernel<8><<<grid, FT, 0, st>>>(g); break;
        default: fsim_ingest_kernel<0><<<grid, FT, 0, st>>>(g); break;
    }
}

// Enqueue FSIM for device-resident pairs; scores[2*i], scores[2*i+1] = FSIM, FSIMc of pair i.
// mma: 0 = FP32 transforms; 1 or 3 = tensor-core transforms with that many products per tile
// (1: FP16 operands, 3: split-precision hi + lo operands) where the plane size has MMA engines.
void fsim_enqueue(iqm_ctx *ctx, const std::vector<iqm_pair> &pairs, int energy_mode, int mma, double *d_scores) {
    const int n_pairs = int(pairs.size());
    // group by plane size, keeping the caller's order inside each group
    std::map<std::pair<int, int>, std::vector<int>> groups;
    std::vector<FsimPairDev> hd(n_pairs);
    for (int i = 0; i < n_pairs; i++) {
        const iqm_pair &q = pairs[i];
        const int F = downscale_factor(q.w, q.h);
        int w2, h2;
        plane_size(q.w, q.h, F, w2, h2);
        IQM_REQUIRE(w2 >= 1 && h2 >= 1, "FSIM plane is empty");
        groups[{w2, h2}].push_back(i);
        hd[i] = FsimPairDev{q.input, q.ref, (long long)q.row_bytes, q.w, q.h, F, i};
    }
    std::vector<FsimPairDev> ordered;
    ordered.reserve(n_pairs);
    for (auto &kv : groups)
        for (int i : kv.second) ordered.push_back(hd[i]);
    auto *d_desc = static_cast<FsimPairDev *>(
        iqm::upload_bytes(ctx, ctx->desc, ordered.data(), sizeof(FsimPairDev) * n_pairs));
    // per-size tables first (building one waits for the context stream)
    struct GroupRun {
        int w2, h2, G, first, slot, F_uniform, chunk;
        int mma;       // tensor-core inverse passes (0: FP32 engines), FP16 intermediate planes
        bool overlap;  // inverse-pass chunks alternate between two streams and two T buffers
        iqm::FsimPlan *P;
        Shapes s;
        Layout L;
        double cost;
    };
    std::vector<GroupRun> runs;
    {
        int first = 0;
        for (auto &kv : groups) {
            GroupRun r{};
            r.w2 = kv.first.first;
            r.h2 = kv.first.second;
            r.G = int(kv.second.size());
            r.first = first;
            r.P = get_plan(ctx, r.w2, r.h2);
            r.s = shapes_for(*r.P, ctx->fsim_tune);
            const int n = r.P->n;
            r.mma = mma_plane(r.w2, r.h2) ? mma : 0;
            if (r.mma) ensure_mma_tables(ctx, r.P);
            const size_t tbytes = r.mma ? sizeof(__half2) : sizeof(float2);
            r.chunk = chunk_pairs(ctx->fsim_tune, r.G, n, tbytes);
            // More than one chunk: split the L2 budget over two buffers and let consecutive chunks run
            // on two streams, so one chunk's column pass fills the other's last partial wave.
            r.overlap = kOverlapChunks && !ctx->timing && r.G > r.chunk;
            if (r.overlap) r.chunk = std::max(1, r.chunk / kChunkStreams);
            r.L = layout_for(r.G, r.chunk, n, int(iqm::ceil_div(n, FT)), r.overlap ? kChunkStreams : 1, tbytes);
            r.F_uniform = hd[kv.second[0]].F;
            for (int i : kv.second)
                if (hd[i].F != r.F_uniform) r.F_uniform = 0;
            r.cost = double(r.G) * n * std::log2(double(n) + 2.0);
            first += r.G;
            runs.push_back(r);
        }
    }
    iqm::timing_mark(ctx, nullptr);
    // Groups are independent: up to kFsimStreams of them run at once on side streams forked from the
    // context stream and joined back (kept on one stream while per-kernel timing is on).  Each
    // stream reuses one scratch slot for its groups, which it runs in order.
    const int S = (runs.size() > 1 && !ctx->timing) ? std::min<int>(int(runs.size()), kFsimStreams) : 1;
    {
        std::vector<int> order(runs.size());
        for (size_t i = 0; i < order.size(); i++) order[i] = int(i);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return runs[a].cost > runs[b].cost; });
        std::vector<double> load(S, 0.0);
        for (int i : order) {
            const int sl = int(std::min_element(load.begin(), load.end()) - load.begin());
            runs[i].slot = sl;
            load[sl] += runs[i].cost;
        }
    }
    std::vector<size_t> slot_off(S + 1, 0);
    {
        std::vector<size_t> need(S, 0);
        for (const auto &r : runs) need[r.slot] = std::max(need[r.slot], r.L.total);
        for (int sl = 0; sl < S; sl++) slot_off[sl + 1] = slot_off[sl] + ((need[sl] + 255) & ~size_t(255));
    }
    auto *base0 = static_cast<uint8_t *>(ctx->scratch.get(slot_off[S], ctx->stream));
    std::vector<cudaStream_t> streams(S, ctx->stream);
    bool any_overlap = false;
    for (const auto &r : runs) any_overlap |= r.overlap;
    if (any_overlap) iqm::side_streams(ctx, kChunkStreams * S);  // streams j*S + slot take chunks k = j mod N
    if (S > 1) {
        iqm::side_streams(ctx, S);
        IQM_CHECK_CUDA(cudaEventRecord(ctx->fork_event, ctx->stream));
        for (int sl = 0; sl < S; sl++) {
            streams[sl] = ctx->side_streams[sl];
            IQM_CHECK_CUDA(cudaStreamWaitEvent(streams[sl], ctx->fork_event, 0));
        }
    }
    for (const GroupRun &r : runs) {
        const int w2 = r.w2, h2 = r.h2, G = r.G;
        iqm::FsimPlan *P = r.P;
        const Shapes &s = r.s;
        cudaStream_t st = streams[r.slot];
        uint8_t *base = base0 + slot_off[r.slot];
        configure_kernels(s);
        const int n = P->n;
        const int tiles = int(iqm::ceil_div(n, FT));
        const int chunk = r.chunk;
        const Layout &Lc = r.L;
        FsimGroup g{};
        g.pairs = d_desc + r.first;
        g.G = G;
        g.pair0 = 0;
        g.w2 = w2;
        g.h2 = h2;
        g.n = n;
        g.yiq = reinterpret_cast<float *>(base + Lc.yiq);
        g.spec = reinterpret_cast<float2 *>(base + Lc.spec);
        g.T = reinterpret_cast<float2 *>(base + Lc.T);
        g.amp = reinterpret_cast<float *>(base + Lc.planes);
        g.energy = g.amp + size_t(G) * 8 * n;
        g.eo0 = g.energy + size_t(G) * 8 * n;
        g.thr = reinterpret_cast<float *>(base + Lc.thr);
        g.partials = reinterpret_cast<double *>(base + Lc.partials);
        g.counters = reinterpret_cast<unsigned *>(base + Lc.counters);
        g.tiles = tiles;
        g.scores = d_scores;
        g.filters = P->filters;
        g.consts = P->consts;
        g.energy_mode = energy_mode;
        IQM_CHECK_CUDA(cudaMemsetAsync(g.counters, 0, sizeof(unsigned) * G, st));
        iqm::timing_mark(ctx, nullptr);
        launch_ingest(g, r.F_uniform, tiles, st);
        iqm::check_launch(ctx, "fsim_ingest_kernel");
        with_engine(s.row_eng, [&](auto e) {
            fsim_fwd_rows_kernel<decltype(e)>
                <<<dim3(iqm::ceil_div(h2, NB << s.lw_rows), G), 32 << s.lw_rows, s.sm_rows, st>>>(g, P->row,
                                                                                                    s.wl_row);
        });
        iqm::check_launch(ctx, "fsim_fwd_rows_kernel");
        with_engine(s.col_eng, [&](auto e) {
            fsim_fwd_cols_kernel<decltype(e)>
                <<<dim3(iqm::ceil_div(w2, NB << s.lw_fcols), G), 32 << s.lw_fcols, s.sm_fcols, st>>>(
                    g, P->col, s.wl_col, s.lw_fcols);
        });
        iqm::check_launch(ctx, "fsim_fwd_cols_kernel");
        // chunk k runs on stream k mod N of this slot (0: the group's stream) with buffer k mod N
        const int nst = r.overlap ? kChunkStreams : 1;
        cudaStream_t cstream[8] = {st};
        if (r.overlap) {
            cudaEvent_t fork = iqm::aux_event(ctx, r.slot);
            IQM_CHECK_CUDA(cudaEventRecord(fork, st));
            for (int j = 1; j < nst; j++) {
                cstream[j] = ctx->side_streams[j * S + r.slot];
                IQM_CHECK_CUDA(cudaStreamWaitEvent(cstream[j], fork, 0));
            }
        }
        for (int c0 = 0, k = 0; c0 < G; c0 += chunk, k++) {
            FsimGroup gc = g;
            gc.pair0 = c0;
            const int j = k % nst;
            cudaStream_t cs = cstream[j];
            const int cg = std::min(chunk, G - c0);
            if (r.mma) {
                gc.Th = reinterpret_cast<__half2 *>(g.T) + size_t(j) * chunk * 32 * n;
                gc.T = nullptr;
                if (r.mma == 3)
                    launch_inv_mma<3>(gc, *P, cg, cs, ctx);
                else
                    launch_inv_mma<1>(gc, *P, cg, cs, ctx);
                continue;
            }
            gc.T = g.T + size_t(j) * chunk * 32 * n;
            launch_inv_cols(gc, *P, s, 2 * cg, 0, cs);
            iqm::check_launch(ctx, "fsim_inv_cols_kernel");
            launch_inv_rows(gc, *P, s, 2 * cg, 0, nullptr, cs);
            iqm::check_launch(ctx, "fsim_inv_rows_kernel");
        }
        for (int j = 1; j < nst; j++) {
            IQM_CHECK_CUDA(cudaEventRecord(ctx->side_events[j * S + r.slot], cstream[j]));
            IQM_CHECK_CUDA(cudaStreamWaitEvent(st, ctx->side_events[j * S + r.slot], 0));
        }
        fsim_noise_kernel<<<dim3(8, G), 1024, 0, st>>>(g);
        iqm::check_launch(ctx, "fsim_noise_kernel");
        if (w2 % 4 == 0)
            fsim_final_kernel<4><<<dim3(int(iqm::ceil_div(n, 4 * FT)), G), FT, 0, st>>>(g);
        else
            fsim_final_kernel<1><<<dim3(tiles, G), FT, 0, st>>>(g);
        iqm::check_launch(ctx, "fsim_final_kernel");
    }
    if (S > 1) {
        for (int sl = 0; sl < S; sl++) {
            IQM_CHECK_CUDA(cudaEventRecord(ctx->side_events[sl], streams[sl]));
            IQM_CHECK_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->side_events[sl], 0));
        }
    }
}

void check_fsim_args(const iqm_pair *pairs, int n, iqm_precision precision, int energy_mode) {
    iqm::check_pairs(pairs, n, 1, 1);
    IQM_REQUIRE(energy_mode == 0 || energy_mode == 1, "energy_mode must be 0 or 1");
    IQM_REQUIRE(precision == IQM_FP32 || precision == IQM_MIXED || precision == IQM_MIXED_FAST, "unknown precision");
    for (int i = 0; i < n; i++) {
        const int F = downscale_factor(pairs[i].w, pairs[i].h);
        int w2, h2;
        plane_size(pairs[i].w, pairs[i].h, F, w2, h2);
        IQM_REQUIRE(w2 >= 2 && h2 >= 2 && w2 <= 4096 && h2 <= 4096,
                    "pair " + std::to_string(i) + ": FSIM plane size out of range");
    }
}

// Products per tensor-core tile of the mixed forms (0: the FP32 form).
int mma_terms(iqm_precision p) { return p == IQM_MIXED ? 3 : p == IQM_MIXED_FAST ? 1 : 0; }

}  // namespace

void iqm_release_fsim_plans(iqm_ctx *ctx) {
    for (auto &kv : ctx->fsim_plans) delete kv.second;
    ctx->fsim_plans.clear();
}

#define IQM_API extern "C" __attribute__((visibility("default")))

void iqm::enqueue_fsim_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n, iqm_precision precision, int energy_mode,
                           double *d_scores) {
    check_fsim_args(pairs, n, precision, energy_mode);
    iqm::check_dev_alignment(pairs, n);
    IQM_REQUIRE(d_scores != nullptr, "d_scores is NULL");
    fsim_enqueue(ctx, std::vector<iqm_pair>(pairs, pairs + n), energy_mode, mma_terms(precision), d_scores);
}

IQM_API int iqm_fsim_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n, iqm_precision precision, int energy_mode,
                         double *d_scores) {
    return iqm::guarded(ctx, [&] { iqm::enqueue_fsim_dev(ctx, pairs, n, precision, energy_mode, d_scores); });
}

IQM_API int iqm_fsim_batch(iqm_ctx *ctx, const iqm_pair *pairs, int n, iqm_precision precision, int energy_mode,
                           double *scores) {
    return iqm::guarded(ctx, [&] {
        check_fsim_args(pairs, n, precision, energy_mode);
        IQM_REQUIRE(scores != nullptr, "scores is NULL");
        auto *d_scores = static_cast<double *>(ctx->scores.get(sizeof(double) * 2 * n, ctx->stream));
        iqm::upload_pipelined(ctx, pairs, n, [&](const iqm_pair *dev, int first, int count) {
            fsim_enqueue(ctx, std::vector<iqm_pair>(dev, dev + count), energy_mode, mma_terms(precision),
                         d_scores + 2 * first);
        });
        IQM_CHECK_CUDA(cudaMemcpyAsync(scores, d_scores, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, ctx->stream));
        IQM_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

IQM_API int iqm_fsim(iqm_ctx *ctx, const uint8_t *rgba_in, const uint8_t *rgba_ref, int w, int h, size_t row_bytes,
                     iqm_precision precision, int energy_mode, double *fsim, double *fsimc) {
    return iqm::guarded(ctx, [&] {
        IQM_REQUIRE(fsim && fsimc, "fsim/fsimc is NULL");
        iqm_pair hp{rgba_in, rgba_ref, w, h, row_bytes};
        check_fsim_args(&hp, 1, precision, energy_mode);
        auto dev = iqm::upload_pairs(ctx, &hp, 1);
        auto *d_scores = static_cast<double *>(ctx->scores.get(sizeof(double) * 2, ctx->stream));
        fsim_enqueue(ctx, dev, energy_mode, mma_terms(precision), d_scores);
        double out[2];
        IQM_CHECK_CUDA(cudaMemcpyAsync(out, d_scores, sizeof(out), cudaMemcpyDeviceToHost, ctx->stream));
        IQM_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
        *fsim = out[0];
        *fsimc = out[1];
    });
}

IQM_API int iqm_fsim_plan_constants(iqm_ctx *ctx, int w2, int h2, int energy_mode, double *em, double *an2,
                                    double *aiaj) {
    return iqm::guarded(ctx, [&] {
        IQM_REQUIRE(w2 >= 2 && h2 >= 2 && w2 <= 4096 && h2 <= 4096, "plane size out of range");
        IQM_REQUIRE(energy_mode == 0 || energy_mode == 1, "energy_mode must be 0 or 1");
        IQM_REQUIRE(em && an2 && aiaj, "output pointer is NULL");
        iqm::FsimPlan *P = get_plan(ctx, w2, h2);
        for (int o = 0; o < 4; o++) {
            em[o] = P->em[o];
            an2[o] = P->an2[energy_mode][o];
            aiaj[o] = P->aiaj[energy_mode][o];
        }
    });
}
