// FLIP (LDR) on sm_100a.
//
// Reference path (cadik/IQM, src/gpu/flip/flip.cpp:121-172, src/gpu/flip/flip_color_pipeline.cpp):
// nine full-image Vulkan dispatches -- sRGB -> YCxCz, feature-filter creation and (racy, in-place)
// normalisation, horizontal and vertical feature passes, horizontal and vertical CSF passes with
// the colour pipeline, colour error, and the combine with a viridis lookup.  The per-pixel value
// pow(dEc, 1 - dEf) is never read back or pooled (FLIPResult::mean_flip is never set); the score
// here is its mean.
//
// Two kernels:
//   flip_hpass_kernel  one CTA per 512-pixel segment of 8 rows of both images, walked row by row
//                      with each row's pixels loaded during the previous row's taps (measured
//                      1.41x the one-row-per-CTA form at 67 ppd): RGBA8 -> linear RGB by a
//                      256-entry table (the sRGB curve of srgb_to_ycxcz.glsl:22-28 on 8-bit inputs),
//                      -> XYZ -> YCxCz in shared memory, then the horizontal feature taps (g, edge,
//                      point on (Y+16)/116, feature_filter_horizontal.glsl) and the horizontal CSF
//                      taps (spatial_prefilter_horizontal.glsl), clamp-to-edge; 4 pixels per thread;
//                      12 planes out;
//   flip_vcols_kernel  (radii known at compile time) 32-column strips, one warp per (image, plane,
//                      filter) role walking down the strip with a (2R+1)-row register window, the
//                      14 filtered values per pixel exchanged through shared memory; or
//   flip_vpass_kernel  (any radii) 32x32-pixel output tiles: the 12 planes (+ halo rows, clamp-to-edge)
//                      staged in shared memory, vertical feature and CSF taps register-blocked 8 rows
//                      per thread; both then YCxCz -> XYZ -> linear RGB (clamped) -> L*a*b* -> Hunt
//                      (spatial_prefilter.glsl:74-99), HyAB colour error (spatial_detection.glsl),
//                      feature error (feature_detection.glsl:48-53), combine
//                      (combine_error_maps.glsl:28) and FP64 pooling; the last CTA of a pair writes
//                      the mean.
// Filter taps depend only on pixels-per-degree: computed on the host in double, normalised once.
// Both images go through the same compiled code (the per-pixel colour math works on float2 pairs
// {input, reference} with packed FP32x2 instructions, the row pass is one loop), so identical
// images give exactly 0.
#include <algorithm>
#include <cmath>
#include <vector>

#include "iqm_internal.cuh"
#include "packed_f32x2.cuh"

#define GLSL_PI 3.141592653589

namespace {

constexpr int MAXR = 32;          // largest supported filter radius (ppd up to ~235)
constexpr int MAXT = 2 * MAXR + 1;
constexpr int HSEG = 512;         // pixels per row segment (hpass)
constexpr int HT = HSEG / 4;      // hpass threads (4 pixels each)
constexpr int HROWS = 8;          // hpass: rows one CTA walks down its segment column
constexpr int HQ = (2 * (HSEG + 2 * MAXR) + HT - 1) / HT;  // staged pixels per thread and row, at most
constexpr int VT_COLS = 32, VT_ROWS = 32, VT_RPT = 8;  // vpass tile and rows per thread
constexpr int VT = VT_COLS * (VT_ROWS / VT_RPT);        // 128 threads
constexpr int NPLANE = 12;        // per pair: [img][dx, ddx, value, Y, Cx, Cz]

struct FlipTaps {
    int rf;               // feature radius: taps j in [-rf, rf] use index j + rf
    int rc;               // CSF radius
    float feat[3][MAXT];  // g, edge, point (normalised as feature_filter_normalize.glsl)
    float csf[3][MAXT];   // luma, red-green, blue-yellow weights, each normalised to sum 1
    float lin[256];       // sRGB byte -> linear
    float rgb2xyz[9], xyz2rgb[9], white[3], inv_white[3];
    float cmax;           // HyAB(Hunt(green), Hunt(blue))^0.7
    float pcc, dec_lo, dec_inv_span;  // 0.4 cmax, 0.95 / pcc, 1 / (cmax - pcc)
};

struct FlipPairDev {
    const uint8_t *a;
    const uint8_t *b;
    float *map;
    long long pitch;
    int w, h;
    int tiles_x, ntiles, tile_base;
    int vec_ok;
    long long plane_off;  // offset (floats) of this pair's 12 planes
    long long seg_base;   // first hpass work unit (HROWS rows of one 512-pixel segment) of this pair
};

struct FlipArgs {
    const FlipPairDev *pairs;
    int npairs;
    float *planes;
    double *partials;
    unsigned *counters;
    double *scores;
    long long total_segs;
};

__device__ __forceinline__ int find_seg(const FlipPairDev *p, int n, long long s) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (p[mid].seg_base <= s) lo = mid; else hi = mid - 1;
    }
    return lo;
}
__device__ __forceinline__ int find_tile(const FlipPairDev *p, int n, int t) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (p[mid].tile_base <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Packed FP32x2 arithmetic for the per-pixel colour terms, whose two halves are the two images.
using iqm::add2;
using iqm::dup2;
using iqm::fma2;
using iqm::mul2;
using iqm::sub2;

// RF, RC > 0: filter radii fixed at compile time (tap loops unrolled, weights as constant-bank
// operands); 0: read from T.
template <int RF, int RC>
__global__ void __launch_bounds__(HT, 8) flip_hpass_kernel(FlipArgs args, const __grid_constant__ FlipTaps T) {
    __shared__ float lin[256];
    __shared__ float ycc[2][4][HSEG + 2 * MAXR];  // Y, Cx, Cz and (Y + 16) / 116
    const long long unit = blockIdx.x;
    const int pi = find_seg(args.pairs, args.npairs, unit);
    const FlipPairDev P = args.pairs[pi];
    const int segs_x = (P.w + HSEG - 1) / HSEG;
    const long long local = unit - P.seg_base;
    const int y_first = int(local / segs_x) * HROWS;
    const int y_end = min(y_first + HROWS, P.h);
    const int x0 = int(local % segs_x) * HSEG;
    const int rf = RF ? RF : T.rf, rc = RC ? RC : T.rc;
    const int R = max(rf, rc);
    for (int i = threadIdx.x; i < 256; i += HT) lin[i] = T.lin[i];
    // columns x0-R .. x0+HSEG+R-1 (clamped to the image) of both images; each thread's share of a
    // row's pixels is loaded a row ahead, so the loads run under the previous row's taps
    const int ncols = HSEG + 2 * R;
    uint32_t raw[HQ];
    auto load_row = [&](int yy) {
#pragma unroll
        for (int k = 0; k < HQ; k++) {
            const int q = threadIdx.x + k * HT;
            if (q < 2 * ncols) {
                const int img = q >= ncols, c = q - img * ncols;  // q < 2 ncols
                const int x = min(max(x0 - R + c, 0), P.w - 1);
                raw[k] = __ldg(reinterpret_cast<const uint32_t *>((img ? P.b : P.a) + (long long)yy * P.pitch) + x);
            }
        }
    };
    load_row(y_first);
    __syncthreads();  // the sRGB table
#pragma unroll 1
    for (int y = y_first; y < y_end; y++) {
    // stage YCxCz of the row, both images
#pragma unroll
    for (int k = 0; k < HQ; k++) {
        const int q = threadIdx.x + k * HT;
        if (q >= 2 * ncols) break;
        const int img = q >= ncols, c = q - img * ncols;  // q < 2 ncols
        const uint32_t px = raw[k];
        const float r = lin[px & 0xffu], g = lin[(px >> 8) & 0xffu], b = lin[(px >> 16) & 0xffu];
        float X = fmaf(T.rgb2xyz[0], r, fmaf(T.rgb2xyz[1], g, T.rgb2xyz[2] * b));
        float Y = fmaf(T.rgb2xyz[3], r, fmaf(T.rgb2xyz[4], g, T.rgb2xyz[5] * b));
        float Z = fmaf(T.rgb2xyz[6], r, fmaf(T.rgb2xyz[7], g, T.rgb2xyz[8] * b));
        X *= T.inv_white[0];
        Y *= T.inv_white[1];
        Z *= T.inv_white[2];
        ycc[img][0][c] = fmaf(116.0f, Y, -16.0f);
        ycc[img][1][c] = 500.0f * (X - Y);
        ycc[img][2][c] = 200.0f * (Y - Z);
        ycc[img][3][c] = (ycc[img][0][c] + 16.0f) * (1.0f / 116.0f);
    }
    __syncthreads();
    if (y + 1 < y_end) load_row(y + 1);
    const int n = P.w * P.h;
    float *planes = args.planes + P.plane_off;
    const int xl = 4 * threadIdx.x;  // first of this thread's 4 segment columns
#pragma unroll 1
    for (int img = 0; img < 2; img++) {
        float fa[4][3] = {}, ca[4][3] = {};
        // output column x = x0 + xl + i, tap j, reads staged column xl + i + u with u = R - j
        if constexpr (RF > 0) {
            // radii known: slide a 4-wide register window along u (one new value per plane per tap)
            constexpr int RR = RF > RC ? RF : RC;
            float win[4][4];
#pragma unroll
            for (int q = 0; q < 4; q++)
#pragma unroll
                for (int i = 0; i < 3; i++) win[q][i + 1] = ycc[img][q][xl + i];
#pragma unroll
            for (int u = 0; u <= 2 * RR; u++) {
#pragma unroll
                for (int q = 0; q < 4; q++) {
#pragma unroll
                    for (int i = 0; i < 3; i++) win[q][i] = win[q][i + 1];
                    win[q][3] = ycc[img][q][xl + u + 3];
                }
                const int j = RR - u;
                if (j >= -RF && j <= RF) {
                    const float wg = T.feat[0][j + RF], we = T.feat[1][j + RF], wp = T.feat[2][j + RF];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        fa[i][0] = fmaf(we, win[3][i], fa[i][0]);  // dx   (edge)
                        fa[i][1] = fmaf(wp, win[3][i], fa[i][1]);  // ddx  (point)
                        fa[i][2] = fmaf(wg, win[3][i], fa[i][2]);  // value (gauss)
                    }
                }
                if (j >= -RC && j <= RC) {
                    const float w0 = T.csf[0][j + RC], w1 = T.csf[1][j + RC], w2 = T.csf[2][j + RC];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        ca[i][0] = fmaf(w0, win[0][i], ca[i][0]);
                        ca[i][1] = fmaf(w1, win[1][i], ca[i][1]);
                        ca[i][2] = fmaf(w2, win[2][i], ca[i][2]);
                    }
                }
            }
        } else {
            for (int j = -R; j <= R; j++) {
                const bool uf = j >= -rf && j <= rf, uc = j >= -rc && j <= rc;
                const float wg = uf ? T.feat[0][j + rf] : 0.f, we = uf ? T.feat[1][j + rf] : 0.f,
                            wp = uf ? T.feat[2][j + rf] : 0.f;
                const float w0 = uc ? T.csf[0][j + rc] : 0.f, w1 = uc ? T.csf[1][j + rc] : 0.f,
                            w2 = uc ? T.csf[2][j + rc] : 0.f;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const int c = xl + i - j + R;
                    const float Yv = ycc[img][0][c];
                    const float v = ycc[img][3][c];
                    fa[i][0] = fmaf(we, v, fa[i][0]);  // dx   (edge)
                    fa[i][1] = fmaf(wp, v, fa[i][1]);  // ddx  (point)
                    fa[i][2] = fmaf(wg, v, fa[i][2]);  // value (gauss)
                    ca[i][0] = fmaf(w0, Yv, ca[i][0]);
                    ca[i][1] = fmaf(w1, ycc[img][1][c], ca[i][1]);
                    ca[i][2] = fmaf(w2, ycc[img][2][c], ca[i][2]);
                }
            }
        }
        const long long p0 = (long long)y * P.w + x0 + xl;
        if ((P.w & 3) == 0 && x0 + xl + 3 < P.w) {
            // 4 consecutive pixels, 16-byte aligned (w, n, plane offsets and xl all multiples of 4)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                *reinterpret_cast<float4 *>(planes + (long long)(img * 6 + c) * n + p0) =
                    make_float4(fa[0][c], fa[1][c], fa[2][c], fa[3][c]);
                *reinterpret_cast<float4 *>(planes + (long long)(img * 6 + 3 + c) * n + p0) =
                    make_float4(ca[0][c], ca[1][c], ca[2][c], ca[3][c]);
            }
        } else {
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int x = x0 + xl + i;
                if (x >= P.w) continue;
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    planes[(long long)(img * 6 + c) * n + p0 + i] = fa[i][c];
                    planes[(long long)(img * 6 + 3 + c) * n + p0 + i] = ca[i][c];
                }
            }
        }
    }
    __syncthreads();  // the row's taps are read before the next row is staged
    }
}

using iqm::cbrt_pos;
using iqm::pow_nonneg;
using iqm::sqrt_nonneg;

// the L*a*b* companding of one normalised XYZ component (shaders/flip/spatial_prefilter.glsl:86-96);
// the shader's pow(v, 1/3) is a cube root
__device__ __forceinline__ float lab_f(float v) {
    const float delta = 6.0f / 29.0f, limit = 0.008856f;
    const float k = 1.0f / (3.0f * delta * delta), o = 4.0f / 29.0f;
    return v > limit ? cbrt_pos(v) : fmaf(v, k, o);
}
__device__ __forceinline__ float2 lab_f2(float2 v) { return make_float2(lab_f(v.x), lab_f(v.y)); }

// filtered YCxCz -> Hunt-adjusted L*a*b* (shaders/flip/spatial_prefilter.glsl:74-99) of both
// images at once
__device__ __forceinline__ void ycxcz_to_hunt_lab2(const FlipTaps &T, float2 Y, float2 Cx, float2 Cz, float2 lab[3]) {
    const float2 yy = mul2(add2(Y, dup2(16.0f)), dup2(1.0f / 116.0f));
    const float2 cx = mul2(Cx, dup2(1.0f / 500.0f)), cz = mul2(Cz, dup2(1.0f / 200.0f));
    const float2 X = mul2(add2(yy, cx), dup2(T.white[0])), Yw = mul2(yy, dup2(T.white[1]));
    const float2 Z = mul2(sub2(yy, cz), dup2(T.white[2]));
    float2 rgb[3];
#pragma unroll
    for (int i = 0; i < 3; i++) {
        const float2 v = fma2(dup2(T.xyz2rgb[3 * i]), X,
                              fma2(dup2(T.xyz2rgb[3 * i + 1]), Yw, mul2(dup2(T.xyz2rgb[3 * i + 2]), Z)));
        rgb[i] = make_float2(fminf(fmaxf(v.x, 0.0f), 1.0f), fminf(fmaxf(v.y, 0.0f), 1.0f));
    }
    float2 c[3];
#pragma unroll
    for (int i = 0; i < 3; i++)
        c[i] = lab_f2(mul2(fma2(dup2(T.rgb2xyz[3 * i]), rgb[0],
                                fma2(dup2(T.rgb2xyz[3 * i + 1]), rgb[1], mul2(dup2(T.rgb2xyz[3 * i + 2]), rgb[2]))),
                           dup2(T.inv_white[i])));
    lab[0] = fma2(dup2(116.0f), c[1], dup2(-16.0f));
    lab[1] = mul2(dup2(500.0f), sub2(c[0], c[1]));
    lab[2] = mul2(dup2(200.0f), sub2(c[1], c[2]));
    const float2 s = mul2(dup2(0.01f), lab[0]);
    lab[1] = mul2(lab[1], s);
    lab[2] = mul2(lab[2], s);
}

// Per-pixel FLIP value from the vertically filtered terms of both images, f[q] = {input,
// reference} of (dx*g, value*edge, ddx*g, value*point, Y*csf0, Cx*csf1, Cz*csf2): feature error
// (feature_detection.glsl:48-53), HyAB colour error of the Hunt-adjusted L*a*b* values
// (spatial_detection.glsl:67-82) and their combination (combine_error_maps.glsl:28).  Each image's
// terms are one half of a packed operation or the same scalar code, so identical images give
// exactly 0.
__device__ __forceinline__ float flip_pixel2(const FlipTaps &T, const float2 (&f)[7]) {
    const float2 g2 = fma2(f[0], f[0], mul2(f[1], f[1])), p2 = fma2(f[2], f[2], mul2(f[3], f[3]));
    float2 lab[3];
    ycxcz_to_hunt_lab2(T, f[4], f[5], f[6], lab);
    const float ed = fabsf(sqrt_nonneg(g2.x) - sqrt_nonneg(g2.y));
    const float pd = fabsf(sqrt_nonneg(p2.x) - sqrt_nonneg(p2.y));
    const float def = sqrt_nonneg(0.70710678f * fmaxf(ed, pd));
    const float d0 = lab[0].x - lab[0].y, d1 = lab[1].x - lab[1].y, d2 = lab[2].x - lab[2].y;
    const float hy = fabsf(d0) + sqrt_nonneg(fmaf(d1, d1, d2 * d2));
    const float de = pow_nonneg(hy, 0.7f);
    const float dec = de < T.pcc ? T.dec_lo * de : 0.95f + ((de - T.pcc) * T.dec_inv_span) * (1.0f - 0.95f);
    return pow_nonneg(dec, 1.0f - def);
}

// the 7 filtered terms of both images from per-image accumulators
__device__ __forceinline__ float flip_pixel(const FlipTaps &T, const float (&f)[2][7]) {
    float2 v[7];
#pragma unroll
    for (int q = 0; q < 7; q++) v[q] = make_float2(f[0][q], f[1][q]);
    return flip_pixel2(T, v);
}

// Pools the CTA's FP64 partial sum; the last CTA of a pair writes the pair's mean.
template <int NT>
__device__ __forceinline__ void pool_tile(const FlipArgs &args, const FlipPairDev &P, int pi, int gt, double dsum,
                                          double *red, int &is_last) {
    for (int d = 16; d > 0; d >>= 1) dsum += __shfl_down_sync(0xffffffffu, dsum, d);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dsum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < NT / 32; i++) t += red[i];
        args.partials[gt] = t;
        __threadfence();
        const unsigned prev = atomicAdd(&args.counters[pi], 1u);
        is_last = prev == unsigned(P.ntiles - 1);
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    double t = 0.0;
    for (int i = threadIdx.x; i < P.ntiles; i += NT) t += __ldcg(&args.partials[P.tile_base + i]);
    for (int d = 16; d > 0; d >>= 1) t += __shfl_down_sync(0xffffffffu, t, d);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double sum = 0.0;
        for (int i = 0; i < NT / 32; i++) sum += red[i];
        args.scores[pi] = sum / (double(P.w) * double(P.h));
        args.counters[pi] = 0u;
    }
}

template <int RF, int RC>
__global__ void __launch_bounds__(VT) flip_vpass_kernel(FlipArgs args, const __grid_constant__ FlipTaps T) {
    extern __shared__ float vs[];  // [NPLANE][rows][VT_COLS]
    __shared__ double red[VT / 32];
    __shared__ int is_last;
    const int gt = blockIdx.x;
    const int pi = find_tile(args.pairs, args.npairs, gt);
    const FlipPairDev P = args.pairs[pi];
    const int local = gt - P.tile_base;
    const int x0 = (local % P.tiles_x) * VT_COLS, y0 = (local / P.tiles_x) * VT_ROWS;
    const int rf = RF ? RF : T.rf, rc = RC ? RC : T.rc;
    const int R = max(rf, rc);
    const int rows = VT_ROWS + 2 * R;
    const int n = P.w * P.h;
    const float *planes = args.planes + P.plane_off;
    // stage rows y0-R .. y0+VT_ROWS+R-1 (clamped), columns x0 .. x0+31 (clamped)
    for (int q = threadIdx.x; q < NPLANE * rows * VT_COLS; q += VT) {
        const int c = q % VT_COLS, r = (q / VT_COLS) % rows, pl = q / (VT_COLS * rows);
        const int y = min(max(y0 - R + r, 0), P.h - 1), x = min(x0 + c, P.w - 1);
        vs[(pl * rows + r) * VT_COLS + c] = planes[(long long)pl * n + (long long)y * P.w + x];
    }
    __syncthreads();
    const int c = threadIdx.x % VT_COLS, rg = threadIdx.x / VT_COLS;
    const int r0 = rg * VT_RPT;  // first output row of this thread within the tile
    // accumulators per output row: per image d(2), dd(2), csf(3)
    float acc[VT_RPT][2][7];
#pragma unroll
    for (int i = 0; i < VT_RPT; i++)
#pragma unroll
        for (int m = 0; m < 2; m++)
#pragma unroll
            for (int q = 0; q < 7; q++) acc[i][m][q] = 0.f;
    // staged row s = r0 + d holds image row y0 - R + s; output row y = y0 + r0 + i reads rows
    // y - k, k in [-r, r], i.e. d = i - k + R.
#pragma unroll
    for (int d = 0; d <= VT_RPT - 1 + 2 * R; d++) {
        const int s = r0 + d;
        float v[2][6];
#pragma unroll
        for (int m = 0; m < 2; m++)
#pragma unroll
            for (int q = 0; q < 6; q++) v[m][q] = vs[((m * 6 + q) * rows + s) * VT_COLS + c];
#pragma unroll
        for (int i = 0; i < VT_RPT; i++) {
            const int k = i - d + R;
            if (k >= -rf && k <= rf) {
                const float g = T.feat[0][k + rf], e = T.feat[1][k + rf], p = T.feat[2][k + rf];
#pragma unroll
                for (int m = 0; m < 2; m++) {
                    acc[i][m][0] = fmaf(v[m][0], g, acc[i][m][0]);  // dx * g
                    acc[i][m][1] = fmaf(v[m][2], e, acc[i][m][1]);  // value * edge
                    acc[i][m][2] = fmaf(v[m][1], g, acc[i][m][2]);  // ddx * g
                    acc[i][m][3] = fmaf(v[m][2], p, acc[i][m][3]);  // value * point
                }
            }
            if (k >= -rc && k <= rc) {
                const float w0 = T.csf[0][k + rc], w1 = T.csf[1][k + rc], w2 = T.csf[2][k + rc];
#pragma unroll
                for (int m = 0; m < 2; m++) {
                    acc[i][m][4] = fmaf(v[m][3], w0, acc[i][m][4]);
                    acc[i][m][5] = fmaf(v[m][4], w1, acc[i][m][5]);
                    acc[i][m][6] = fmaf(v[m][5], w2, acc[i][m][6]);
                }
            }
        }
    }
    double dsum = 0.0;
    const int x = x0 + c;
#pragma unroll
    for (int i = 0; i < VT_RPT; i++) {
        const int y = y0 + r0 + i;
        if (x >= P.w || y >= P.h) continue;
        const float val = flip_pixel(T, acc[i]);
        if (P.map) P.map[(long long)y * P.w + x] = val;
        dsum += double(val);
    }
    pool_tile<VT>(args, P, pi, gt, dsum, red, is_last);
}

// ---------------------------------------------------------------------------------------------
// Vertical pass for compile-time radii ("column walkers").  Warp w of a CTA runs role w -- one
// (image, plane, filter) combination -- down the CTA's 32 columns over CW_BLOCKS blocks of
// K = 2R+1 rows, keeping the last K rows of its plane in a register window whose slots are fixed
// at compile time (slot = input row mod K), so each output row costs one coalesced load and the
// filter's FMAs.  After every block the CTA turns the 14 filtered values of each of its K x 32
// pixels into FLIP values (flip_pixel) from a shared-memory buffer.
constexpr int CW_ROLES = 14;         // per image: dx*g, value*edge, ddx*g, value*point, Y*csf0, Cx*csf1, Cz*csf2
constexpr int CW_T = 32 * CW_ROLES;  // 448 threads
constexpr int CW_BLOCKS = 10;        // K-row blocks per CTA
constexpr int CW_GROUP = 2;          // blocks filtered before each pixel phase (2 x 21 x 32 = 3 pixels a thread)
static_assert(CW_BLOCKS % CW_GROUP == 0, "a CTA's blocks split into whole groups");

__host__ __device__ constexpr int cw_rows(int rf, int rc) { return CW_BLOCKS * (2 * (rf > rc ? rf : rc) + 1); }

// One block of K output rows: window slot (j + u) % K holds image row y - R + u of output row
// y = ybase + R + j, weighted by taps[u].  Every role runs this one body (one copy of the unrolled
// code for all warps); a role whose filter is shorter than K has zero taps at the ends, which leave
// its sums unchanged bit for bit.
template <int K>
__device__ __forceinline__ void cw_block(float (&win)[K], const float (&taps)[K], const float *col, int w, int h,
                                         int ybase, float *out) {
#pragma unroll
    for (int j = 0; j < K; j++) {
        const int y = min(max(ybase + j + K - 1, 0), h - 1);
        win[(j + K - 1) % K] = __ldg(col + size_t(y) * size_t(w));
        float acc = 0.f;
#pragma unroll
        for (int u = 0; u < K; u++) acc = fmaf(win[(j + u) % K], taps[u], acc);
        out[j * CW_ROLES * 32] = acc;
    }
}

template <int RF, int RC>
__global__ void __launch_bounds__(CW_T, 2) flip_vcols_kernel(FlipArgs args, const __grid_constant__ FlipTaps T) {
    constexpr int R = RF > RC ? RF : RC;
    constexpr int K = 2 * R + 1;
    constexpr int SEG = cw_rows(RF, RC);
    extern __shared__ float cw_buf[];  // [CW_GROUP * K rows][CW_ROLES][32 columns]
    __shared__ double red[CW_T / 32];
    __shared__ int is_last;
    const int gt = blockIdx.x;
    const int pi = find_tile(args.pairs, args.npairs, gt);
    const FlipPairDev P = args.pairs[pi];
    const int local = gt - P.tile_base;
    const int x0 = (local % P.tiles_x) * 32, y0 = (local / P.tiles_x) * SEG;
    const int lane = threadIdx.x & 31, role = threadIdx.x >> 5;
    const int f = role % 7, m = role / 7;
    // plane of each role within the image's six: dx, ddx, value, Y, Cx, Cz
    const int pl = m * 6 + (f == 0 ? 0 : f == 1 ? 2 : f == 2 ? 1 : f == 3 ? 2 : f - 1);
    const size_t n = size_t(P.w) * size_t(P.h);
    const float *col = args.planes + P.plane_off + size_t(pl) * n + min(x0 + lane, P.w - 1);
    // this role's taps: image row y - k weighs tap k + radius; feature roles use g, edge, g, point
    const float *tap_src = f < 4 ? T.feat[f == 1 ? 1 : f == 3 ? 2 : 0] : T.csf[f - 4];
    const int rad = f < 4 ? RF : RC;
    float win[K];
#pragma unroll
    for (int t = 0; t < K - 1; t++) win[t] = __ldg(col + size_t(min(max(y0 - R + t, 0), P.h - 1)) * size_t(P.w));
    float *out = cw_buf + role * 32 + lane;
    double dsum = 0.0;
    for (int b = 0; b < CW_BLOCKS; b += CW_GROUP) {
        const int yg = y0 + b * K;
        if (yg >= P.h) break;  // uniform over the CTA
        for (int bb = 0; bb < CW_GROUP; bb++) {
            const int yb = yg + bb * K;
            if (yb >= P.h) break;  // uniform; rows past the image are skipped by the pixel phase
            float taps[K];  // reloaded per block so they are not live across the pixel phase
#pragma unroll
            for (int u = 0; u < K; u++) {
                const int k = R - u;
                taps[u] = (k >= -rad && k <= rad) ? tap_src[k + rad] : 0.f;
            }
            cw_block<K>(win, taps, col, P.w, P.h, yb - R, out + bb * K * CW_ROLES * 32);
        }
        __syncthreads();
        for (int p = threadIdx.x; p < CW_GROUP * K * 32; p += CW_T) {
            const int j = p >> 5, c = p & 31;
            const int y = yg + j, x = x0 + c;
            if (y >= P.h || x >= P.w) continue;
            float v[2][7];
            const float *px = cw_buf + j * CW_ROLES * 32 + c;
#pragma unroll
            for (int mm = 0; mm < 2; mm++)
#pragma unroll
                for (int q = 0; q < 7; q++) v[mm][q] = px[(mm * 7 + q) * 32];
            const float val = flip_pixel(T, v);
            if (P.map) P.map[size_t(y) * size_t(P.w) + x] = val;
            dsum += double(val);
        }
        __syncthreads();
    }
    pool_tile<CW_T>(args, P, pi, gt, dsum, red, is_last);
}

// ---------------------------------------------------------------------------------------------
// host side

double ppd_of(const iqm_flip_params &p) {  // src/gpu/flip/flip.cpp:125 (float operands)
    const float f = p.monitor_distance * (p.monitor_resolution_x / p.monitor_width);
    return double(f) * (M_PI / 180.0);
}

void make_taps(double ppd, FlipTaps &T) {
    // feature taps: shaders/flip/feature_filter.glsl:26-37 with the kernel size of flip.cpp:126,
    // then feature_filter_normalize.glsl:27-46 (positive and negative parts normalised separately)
    const float ppdf = float(ppd);
    const int K = 2 * int(std::ceil(3 * 0.5 * 0.082 * ppd)) + 1;
    const double sd = 0.5 * 0.082 * double(ppdf);
    const int radius = int(std::ceil(3.0f * float(0.5f * 0.082f * ppdf)));
    IQM_REQUIRE(K / 2 <= MAXR, "pixels per degree too large for the FLIP filters");
    T.rf = K / 2;
    std::vector<double> t[3];
    for (int c = 0; c < 3; c++) t[c].assign(K, 0.0);
    double pos[3] = {0, 0, 0}, neg[3] = {0, 0, 0};
    for (int x = 0; x < K; x++) {
        const double xc = double(x - radius);
        const double g = std::exp(-(xc * xc) / (2.0 * sd * sd));
        t[0][x] = g;
        t[1][x] = -xc * g;
        t[2][x] = (xc * xc / (sd * sd) - 1.0) * g;
        for (int c = 0; c < 3; c++) (t[c][x] > 0 ? pos[c] : neg[c]) += std::fabs(t[c][x]);
    }
    for (int c = 0; c < 3; c++)
        for (int x = 0; x < MAXT; x++)
            T.feat[c][x] = x < K ? float(t[c][x] > 0 ? t[c][x] / pos[c] : t[c][x] / neg[c]) : 0.f;
    // CSF taps: shaders/flip/spatial_prefilter_horizontal.glsl:20-61
    const double pi = GLSL_PI;
    const int rc = int(std::ceil(3.0f * std::sqrt(0.04f / (2.0f * float(pi) * float(pi))) * ppdf));
    IQM_REQUIRE(rc <= MAXR, "pixels per degree too large for the FLIP filters");
    T.rc = rc;
    const double par[3][4] = {{1.0, 0.0047, 0, 0.00001}, {1.0, 0.0053, 0, 0.00001}, {34.1, 0.04, 13.5, 0.025}};
    const double dx = 1.0 / double(ppdf);
    for (int ch = 0; ch < 3; ch++) {
        std::vector<double> w(2 * rc + 1);
        double tot = 0;
        for (int j = -rc; j <= rc; j++) {
            const double d = (j * dx) * (j * dx);
            const double* q = par[ch];
            w[j + rc] = q[0] * std::sqrt(pi / q[1]) * std::exp(-pi * pi * d / q[1]) +
                        q[2] * std::sqrt(pi / q[3]) * std::exp(-pi * pi * d / q[3]);
            tot += w[j + rc];
        }
        for (int j = 0; j < MAXT; j++) T.csf[ch][j] = j < 2 * rc + 1 ? float(w[j] / tot) : 0.f;
    }
    // sRGB -> linear for every byte value (srgb_to_ycxcz.glsl:22-28)
    for (int i = 0; i < 256; i++) {
        const float c = float(i) / 255.0f;
        T.lin[i] = c > 0.04045f ? std::pow((c + 0.055f) / 1.055f, 2.4f) : c / 12.92f;
    }
    // RGB_TO_XYZ (srgb_to_ycxcz.glsl:16-20), XYZ_TO_RGB (spatial_prefilter.glsl:20-24): GLSL mat3
    // is column-major and `v * M` dots v with each column, so row i below is column i there.
    const double m[9] = {10135552.0 / 24577794, 8788810.0 / 24577794, 4435075.0 / 24577794,
                         2613072.0 / 12288897, 8788810.0 / 12288897, 887015.0 / 12288897,
                         1425312.0 / 73733382, 8788810.0 / 73733382, 70074185.0 / 73733382};
    const double mi[9] = {3.241003275, -1.537398934, -0.498615861, -0.969224334, 1.875930071,
                          0.041554224, 0.055639423, -0.204011202, 1.057148933};
    for (int i = 0; i < 9; i++) {
        T.rgb2xyz[i] = float(m[i]);
        T.xyz2rgb[i] = float(mi[i]);
    }
    for (int i = 0; i < 3; i++) {
        T.white[i] = T.rgb2xyz[3 * i] + T.rgb2xyz[3 * i + 1] + T.rgb2xyz[3 * i + 2];
        T.inv_white[i] = 1.0f / T.white[i];
    }
    // cmax = HyAB(Hunt(green), Hunt(blue))^0.7 (spatial_detection.glsl:73-81), host double
    auto lab_of = [&](double r, double g, double b, double lab[3]) {
        double xyz[3];
        for (int i = 0; i < 3; i++) xyz[i] = (m[3 * i] * r + m[3 * i + 1] * g + m[3 * i + 2] * b) / double(T.white[i]);
        const double delta = 6.0 / 29.0, lim = 0.008856;
        double c[3];
        for (int i = 0; i < 3; i++) c[i] = xyz[i] > lim ? std::cbrt(xyz[i]) : xyz[i] / (3 * delta * delta) + 4.0 / 29.0;
        lab[0] = 116 * c[1] - 16;
        lab[1] = 500 * (c[0] - c[1]) * 0.01 * lab[0];
        lab[2] = 200 * (c[1] - c[2]) * 0.01 * lab[0];
    };
    double lg[3], lb[3];
    lab_of(0, 1, 0, lg);
    lab_of(0, 0, 1, lb);
    const double hy = std::fabs(lg[0] - lb[0]) + std::sqrt((lg[1] - lb[1]) * (lg[1] - lb[1]) + (lg[2] - lb[2]) * (lg[2] - lb[2]));
    T.cmax = float(std::pow(hy, 0.7));
    T.pcc = 0.4f * T.cmax;
    T.dec_lo = 0.95f / T.pcc;
    T.dec_inv_span = 1.0f / (T.cmax - T.pcc);
}

iqm_flip_params resolve(const iqm_flip_params *p) {
    iqm_flip_params d;
    iqm_flip_default_params(&d);
    return p ? *p : d;
}

void check_params(const iqm_flip_params &p) {
    IQM_REQUIRE(std::isfinite(p.monitor_resolution_x) && std::isfinite(p.monitor_distance) &&
                    std::isfinite(p.monitor_width) && p.monitor_resolution_x > 0 && p.monitor_distance > 0 &&
                    p.monitor_width > 0,
                "FLIP monitor parameters must be positive");
}

void flip_enqueue(iqm_ctx *ctx, const std::vector<iqm_pair> &pairs, const iqm_flip_params &params,
                  const std::vector<float *> &maps, double *d_scores) {
    FlipTaps T{};
    make_taps(ppd_of(params), T);
    const int n = int(pairs.size());
    // the two viewing set-ups in common use get kernels with their radii built in
    const int fixed = (T.rf == 7 && T.rc == 8) ? 1 : (T.rf == 9 && T.rc == 10) ? 2 : 0;
    const int tile_rows = fixed == 1 ? cw_rows(7, 8) : fixed == 2 ? cw_rows(9, 10) : VT_ROWS;
    std::vector<FlipPairDev> hd(n);
    long long segs = 0, plane_floats = 0;
    int tiles = 0;
    for (int i = 0; i < n; i++) {
        const iqm_pair &q = pairs[i];
        FlipPairDev &d = hd[i];
        d.a = q.input;
        d.b = q.ref;
        d.map = maps.empty() ? nullptr : maps[i];
        d.pitch = (long long)q.row_bytes;
        d.w = q.w;
        d.h = q.h;
        d.tiles_x = int(iqm::ceil_div(q.w, VT_COLS));
        d.ntiles = d.tiles_x * int(iqm::ceil_div(q.h, tile_rows));
        d.tile_base = tiles;
        d.vec_ok = 0;
        d.plane_off = plane_floats;
        d.seg_base = segs;
        tiles += d.ntiles;
        segs += (long long)iqm::ceil_div(q.w, HSEG) * iqm::ceil_div(q.h, HROWS);
        plane_floats += (long long)NPLANE * q.w * q.h;
    }
    IQM_REQUIRE(segs < (1LL << 31) && tiles < (1 << 30), "batch too large");
    auto *d_desc = static_cast<FlipPairDev *>(iqm::upload_bytes(ctx, ctx->desc, hd.data(), sizeof(FlipPairDev) * n));
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t pb = al(sizeof(float) * size_t(plane_floats)), qb = al(sizeof(double) * tiles),
                 cb = al(sizeof(unsigned) * n);
    auto *base = static_cast<uint8_t *>(ctx->scratch.get(pb + qb + cb, ctx->stream));
    FlipArgs a{};
    a.pairs = d_desc;
    a.npairs = n;
    a.planes = reinterpret_cast<float *>(base);
    a.partials = reinterpret_cast<double *>(base + pb);
    a.counters = reinterpret_cast<unsigned *>(base + pb + qb);
    a.scores = d_scores;
    a.total_segs = segs;
    IQM_CHECK_CUDA(cudaMemsetAsync(a.counters, 0, sizeof(unsigned) * n, ctx->stream));
    iqm::timing_mark(ctx, nullptr);
    const int R = std::max(T.rf, T.rc);
    const size_t smem = sizeof(float) * NPLANE * (VT_ROWS + 2 * R) * VT_COLS;
    // dynamic shared memory of the column walkers: CW_GROUP blocks of K rows x 14 roles x 32 columns
    auto cw_smem = [](int rf, int rc) { return sizeof(float) * CW_GROUP * (2 * std::max(rf, rc) + 1) * CW_ROLES * 32; };
    if (fixed == 1) {  // default monitor, 52.1 ppd
        flip_hpass_kernel<7, 8><<<unsigned(segs), HT, 0, ctx->stream>>>(a, T);
        iqm::check_launch(ctx, "flip_hpass_kernel");
        const size_t sm = cw_smem(7, 8);
        IQM_CHECK_CUDA(cudaFuncSetAttribute((const void *)flip_vcols_kernel<7, 8>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
        flip_vcols_kernel<7, 8><<<tiles, CW_T, sm, ctx->stream>>>(a, T);
        iqm::check_launch(ctx, "flip_vcols_kernel");
    } else if (fixed == 2) {  // 67 ppd
        flip_hpass_kernel<9, 10><<<unsigned(segs), HT, 0, ctx->stream>>>(a, T);
        iqm::check_launch(ctx, "flip_hpass_kernel");
        const size_t sm = cw_smem(9, 10);
        IQM_CHECK_CUDA(cudaFuncSetAttribute((const void *)flip_vcols_kernel<9, 10>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
        flip_vcols_kernel<9, 10><<<tiles, CW_T, sm, ctx->stream>>>(a, T);
        iqm::check_launch(ctx, "flip_vcols_kernel");
    } else {
        flip_hpass_kernel<0, 0><<<unsigned(segs), HT, 0, ctx->stream>>>(a, T);
        iqm::check_launch(ctx, "flip_hpass_kernel");
        if (smem > 48 * 1024)
            IQM_CHECK_CUDA(cudaFuncSetAttribute((const void *)flip_vpass_kernel<0, 0>,
                                                cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        flip_vpass_kernel<0, 0><<<tiles, VT, smem, ctx->stream>>>(a, T);
        iqm::check_launch(ctx, "flip_vpass_kernel");
    }
}

}  // namespace

#define IQM_API extern "C" __attribute__((visibility("default")))

IQM_API void iqm_flip_default_params(iqm_flip_params *p) {
    if (!p) return;
    // src/gpu/flip/flip.h:21-25
    p->monitor_resolution_x = 2560.f;
    p->monitor_distance = 0.7f;
    p->monitor_width = 0.6f;
}

IQM_API double iqm_flip_ppd(const iqm_flip_params *p) { return ppd_of(resolve(p)); }

void iqm::enqueue_flip_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n, const iqm_flip_params *params,
                           double *d_scores) {
    const iqm_flip_params p = resolve(params);
    check_params(p);
    iqm::check_pairs(pairs, n, 1, 1);
    iqm::check_dev_alignment(pairs, n);
    IQM_REQUIRE(d_scores != nullptr, "d_scores is NULL");
    flip_enqueue(ctx, std::vector<iqm_pair>(pairs, pairs + n), p, {}, d_scores);
}

IQM_API int iqm_flip_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n, const iqm_flip_params *params,
                         double *d_scores) {
    return iqm::guarded(ctx, [&] { iqm::enqueue_flip_dev(ctx, pairs, n, params, d_scores); });
}

IQM_API int iqm_flip_batch(iqm_ctx *ctx, const iqm_pair *pairs, int n, const iqm_flip_params *params,
                           double *scores) {
    return iqm::guarded(ctx, [&] {
        const iqm_flip_params p = resolve(params);
        check_params(p);
        iqm::check_pairs(pairs, n, 1, 1);
        IQM_REQUIRE(scores != nullptr, "scores is NULL");
        auto *d_scores = static_cast<double *>(ctx->scores.get(sizeof(double) * n, ctx->stream));
        iqm::upload_pipelined(ctx, pairs, n, [&](const iqm_pair *dev, int first, int count) {
            flip_enqueue(ctx, std::vector<iqm_pair>(dev, dev + count), p, {}, d_scores + first);
        });
        IQM_CHECK_CUDA(cudaMemcpyAsync(scores, d_scores, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
        IQM_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

IQM_API int iqm_flip(iqm_ctx *ctx, const uint8_t *rgba_in, const uint8_t *rgba_ref, int w, int h, size_t row_bytes,
                     const iqm_flip_params *params, float *err_map, double *mean_flip) {
    return iqm::guarded(ctx, [&] {
        const iqm_flip_params p = resolve(params);
        check_params(p);
        IQM_REQUIRE(mean_flip != nullptr, "mean_flip is NULL");
        iqm_pair hp{rgba_in, rgba_ref, w, h, row_bytes};
        iqm::check_pairs(&hp, 1, 1, 1);
        auto dev = iqm::upload_pairs(ctx, &hp, 1);
        auto *d_score = static_cast<double *>(ctx->scores.get(sizeof(double), ctx->stream));
        std::vector<float *> maps;
        float *d_map = nullptr;
        if (err_map) {
            d_map = static_cast<float *>(ctx->maps.get(sizeof(float) * size_t(w) * h, ctx->stream));
            maps.push_back(d_map);
        }
        flip_enqueue(ctx, dev, p, maps, d_score);
        IQM_CHECK_CUDA(cudaMemcpyAsync(mean_flip, d_score, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        if (err_map)
            IQM_CHECK_CUDA(cudaMemcpyAsync(err_map, d_map, sizeof(float) * size_t(w) * h, cudaMemcpyDeviceToHost,
                                           ctx->stream));
        IQM_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}
