// SSIM with the Gaussian window sums on the tensor cores (IQM_MIXED, IQM_MIXED_FAST).
//
// Included by ssim.cu (it uses SsimPairDev, find_pair and pool_tiles from there).  The quantities
// are those of the FP32 kernel -- the four moments of u = a + b and v = a - b about a per-tile
// shift, the in-image truncated window renormalised per pixel, MSSIM over x, y in [R, dim - R] --
// with the two 1-D window passes run as banded matrix products (mma.sync m16n8k16, FP16 operands,
// FP32 accumulation):
//
//   horizontal  Ht[c][y] = sum_j Gb[c][j] M[y][x0 - 8 + j]   (c: 16 output columns, j: 32 inputs)
//   vertical    S[r][c]  = sum_k Gb[r][k] H[y0 - 8 + k][c]   (r: 16 output rows,    k: 32 H rows)
//
// with Gb[m][j] = g(j - 8 - m) (the normalised 1-D Gaussian, zero beyond its radius R <= 7, so
// 16 + 2R <= 32 inputs cover 16 outputs).  The same band matrix is the A operand of both passes.
// The horizontal pass is computed transposed (output columns as rows of the product), so its
// accumulators -- m16n8 C fragments of (column, row) -- are, packed to FP16 pairs, exactly the
// B fragments of the vertical product (k = image row, n = column): the horizontal results never
// leave registers.  The moments enter the horizontal pass from shared memory through ldmatrix.
//
// CTA tile: 64 output columns (4 warps x 16) x 64 output rows (four 16-row blocks); the CTA works
// from image rows y0-8 .. y0+71 and columns x0-8 .. x0+71 (1.56 staged pixels per output pixel).
// The kernel is persistent: each CTA walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ...  Per
// tile: load the RGBA8 rows and stage them as FP16 moment planes (one barrier), then each warp runs
// its five 16-row horizontal blocks and four vertical blocks in a rolled loop (the code stays in
// the instruction cache).  The moments are taken about the tile's centre pixel (u, v) and scaled
// by 2^12 (largest staged magnitude 4 * 2^12, well inside FP16's range, and small values stay clear
// of FP16's subnormals).  The split form walks column segments of six tiles with one shift per
// segment (its accuracy does not depend on the shift tile): each later tile reuses the previous
// tile's last horizontal block from registers and stages 64 rows, not 80.  Measured at 1080p
// (17 tiles a column) with segments of 4 / 5 / 6 / 7 / 8 tiles: 0.96 / 1.06 / 1.08 / 1.02 / 0.99x
// the FP32 kernel.
// Measured against 64x32 tiles, the taller tile stages a third fewer pixels
// per output and runs 1.35x faster despite one CTA fewer per SM; taller or wider tiles were slower
// (96 or 128 rows) or took the single-product form past its bound (128 columns).
//
// IQM_MIXED stages every moment as an FP16 hi + lo pair and forms each product as
// A_hi B_hi + A_hi B_lo + A_lo B_hi (about 21 significant bits, MSSIM within ~1e-6 of FP64);
// IQM_MIXED_FAST uses the hi parts alone (11-bit moments and taps: MSSIM within a few 1e-5 of FP64
// on large images, tested to 2e-4; the error grows with how far a tile's pixels lie from its
// centre pixel, which bounds the tile's size).  The per-pixel weight normalisation uses the window
// as the tensor cores see it (FP16-rounded taps in the fast form).
#pragma once

#include "dft_mma.cuh"

namespace {

constexpr int MT_W = 64;              // output columns per CTA tile (a multiple of 16)
constexpr int MT_H = 64;              // output rows per CTA tile (a multiple of 16)
constexpr int MT_THREADS = 2 * MT_W;  // one warp per 16 output columns
constexpr int MT_ROWS = MT_H + 16;    // staged rows y0-8 .. y0+MT_H+7 (MT_H/16 + 1 horizontal blocks)
constexpr int MT_SCOLS = MT_W + 16;   // staged columns x0-8 .. x0+MT_W+7
constexpr int MT_LD = MT_SCOLS + 8;   // FP16 row stride of a staged plane: 48 mod 128 bytes, so the 8
                                      // rows of one ldmatrix 8x8 load fall in distinct 16-byte groups
static_assert((2 * MT_LD) % 128 == 48, "ldmatrix rows must fall in distinct bank groups");
// CTAs per SM the launch bounds ask for: shared memory allows 3 (single products, 56 KB a CTA) and
// 2 (split products, 112 KB); the register budgets follow.
constexpr int MT_MIN_CTAS_SINGLE = 512 / MT_THREADS, MT_MIN_CTAS_SPLIT = 256 / MT_THREADS > 0 ? 256 / MT_THREADS : 1;
constexpr float MT_SCALE = 4096.f;    // staged moments are scaled by 2^12
constexpr int MT_SEG_SPLIT = 6;       // tiles per column segment (a work unit; the split form's shift tile)

struct SsimMmaArgs {
    const SsimPairDev *pairs;
    int npairs;
    int R;               // window radius, 1..7
    double *partials;    // one per tile
    unsigned *counters;  // one per pair, zero on entry
    double *scores;      // one per pair
    float gn[15];        // g(-R..R) / sum g, zero beyond 2R
    float c1, c2;
};

template <int SPLIT>
struct SsimMmaGeom {
    static constexpr int PLANES = SPLIT == 1 ? 4 : 8;  // su, sv, su^2, sv^2 (hi), then their lo parts
    static constexpr int PLANE = MT_ROWS * MT_LD;      // halves per plane
    static constexpr size_t smem_bytes = size_t(PLANES) * PLANE * 2;
};

__device__ __forceinline__ void ldmatrix_x4(unsigned (&r)[4], const void *p) {
    const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a));
}

// Byte k of two RGBA8 words as exact floats: each byte placed under the exponent of 2^23 (an
// integer-pipe byte permute), then 2^23 subtracted from both at once (instead of the quarter-rate
// integer-to-float conversion).
template <int K>
__device__ __forceinline__ float2 bytes_f2(uint32_t pa, uint32_t pb) {
    const float2 f = make_float2(__uint_as_float(__byte_perm(pa, 0x4B000000u, 0x7540 + K)),
                                 __uint_as_float(__byte_perm(pb, 0x4B000000u, 0x7540 + K)));
    return __fadd2_rn(f, make_float2(-8388608.0f, -8388608.0f));
}

// The two lumas of a pixel pair, shaders/ssim/ssim_lumapack.glsl:19-21 on unorm bytes.
__device__ __forceinline__ float2 luma2(uint32_t pa, uint32_t pb) {
    const float2 r = bytes_f2<0>(pa, pb);
    const float2 g = bytes_f2<1>(pa, pb);
    const float2 b = bytes_f2<2>(pa, pb);
    const float s = 1.0f / 255.0f;
    float2 l = __fmul2_rn(make_float2(0.114f * s, 0.114f * s), b);
    l = __ffma2_rn(make_float2(0.581f * s, 0.581f * s), g, l);
    return __ffma2_rn(make_float2(0.299f * s, 0.299f * s), r, l);
}

// Stage the tile's moment planes: staged row r = image row y0 - 8 + r, staged column q = image column
// x0 - 8 + q; positions outside the image hold zero in every plane (they drop out of the sums).
// The thread's loads are issued in two rounds of up to seven 4-pixel chunks (fourteen 16-byte loads
// in flight per thread) ahead of their conversion: two memory round trips per tile, with the code
// of one round only.  (Prefetching the next tile into shared memory instead hides the round trips but
// costs a CTA per SM, which measured slower.)
template <int SPLIT>
__device__ __forceinline__ void stage_moments(__half *pl, const SsimPairDev &P, int x0, int y0, float cu, float cv,
                                              int row_lo) {
    using G = SsimMmaGeom<SPLIT>;
    constexpr int CH = MT_SCOLS / 4;  // 4-pixel chunks per staged row
    constexpr int PER_T = (MT_ROWS * CH + MT_THREADS - 1) / MT_THREADS;
    constexpr int HALF = (PER_T + 1) / 2;
    const int CHUNKS = (MT_ROWS - row_lo) * CH;  // staged rows row_lo .. MT_ROWS - 1
#pragma unroll 1
    for (int k0 = 0; k0 < PER_T; k0 += HALF) {
        uint4 ra[HALF], rb[HALF];
#pragma unroll
        for (int kk = 0; kk < HALF; kk++) {
            const int c = threadIdx.x + (k0 + kk) * MT_THREADS;
            const int r = row_lo + c / CH, q = c % CH;
            const int y = y0 - 8 + r, x = x0 - 8 + 4 * q;  // x is a multiple of 4: a chunk is all in or all left of 0
            ra[kk] = make_uint4(0u, 0u, 0u, 0u);
            rb[kk] = make_uint4(0u, 0u, 0u, 0u);
            if (c < CHUNKS && y >= 0 && y < P.h && x >= 0 && x < P.w) {
                const int nv = min(4, P.w - x);
                const uint8_t *pa = P.a + (long long)y * P.pitch + 4LL * x;
                const uint8_t *pb = P.b + (long long)y * P.pitch + 4LL * x;
                if (P.vec_ok && nv == 4) {
                    ra[kk] = __ldg(reinterpret_cast<const uint4 *>(pa));
                    rb[kk] = __ldg(reinterpret_cast<const uint4 *>(pb));
                } else {
                    const uint32_t *wa = reinterpret_cast<const uint32_t *>(pa);
                    const uint32_t *wb = reinterpret_cast<const uint32_t *>(pb);
                    ra[kk].x = __ldg(wa);
                    rb[kk].x = __ldg(wb);
                    if (nv > 1) ra[kk].y = __ldg(wa + 1), rb[kk].y = __ldg(wb + 1);
                    if (nv > 2) ra[kk].z = __ldg(wa + 2), rb[kk].z = __ldg(wb + 2);
                    if (nv > 3) ra[kk].w = __ldg(wa + 3), rb[kk].w = __ldg(wb + 3);
                }
            }
        }
#pragma unroll
        for (int kk = 0; kk < HALF; kk++) {
            const int c = threadIdx.x + (k0 + kk) * MT_THREADS;
            if (c >= CHUNKS) break;
            const int r = row_lo + c / CH, q = c % CH;
            const int y = y0 - 8 + r, x = x0 - 8 + 4 * q;
            const int nv = (y >= 0 && y < P.h && x >= 0) ? min(4, P.w - x) : 0;
            const uint32_t a[4] = {ra[kk].x, ra[kk].y, ra[kk].z, ra[kk].w};
            const uint32_t b[4] = {rb[kk].x, rb[kk].y, rb[kk].z, rb[kk].w};
            float m[4][4];  // [moment][pixel]: su, sv, su^2, sv^2 (scaled)
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const float2 l = luma2(a[i], b[i]);
                // (du, dv) = (la + lb - cu, la - lb - cv); sm = (du, dv) * 2^12; sq = (du, dv) * sm
                const float2 d = __ffma2_rn(make_float2(l.y, l.y), make_float2(1.f, -1.f),
                                            __fadd2_rn(make_float2(l.x, l.x), make_float2(-cu, -cv)));
                float2 sm = __fmul2_rn(d, make_float2(MT_SCALE, MT_SCALE));
                if (i >= nv) sm = make_float2(0.f, 0.f);  // outside the image
                const float2 sq = __fmul2_rn(d, sm);
                m[0][i] = sm.x;
                m[1][i] = sm.y;
                m[2][i] = sq.x;
                m[3][i] = sq.y;
            }
            const int off = r * MT_LD + 4 * q;
#pragma unroll
            for (int p = 0; p < 4; p++) {
                if (SPLIT == 1) {
                    *reinterpret_cast<uint2 *>(pl + p * G::PLANE + off) =
                        make_uint2(iqm::pack_h2(m[p][0], m[p][1]), iqm::pack_h2(m[p][2], m[p][3]));
                } else {
                    unsigned h0, l0, h1, l1;
                    iqm::split_h2(m[p][0], m[p][1], h0, l0);
                    iqm::split_h2(m[p][2], m[p][3], h1, l1);
                    *reinterpret_cast<uint2 *>(pl + p * G::PLANE + off) = make_uint2(h0, h1);
                    *reinterpret_cast<uint2 *>(pl + (p + 4) * G::PLANE + off) = make_uint2(l0, l1);
                }
            }
        }
    }
}

// One 16-row horizontal block (staged rows 16 hb .. 16 hb + 15) of this warp's 16 columns, as the
// vertical pass's B fragments: hh[p][v][kb] (moment p, output columns 8v..8v+7, block rows
// 8kb..8kb+7 as the fragment's k rows 2t, 2t+1 (+8)); hl the lo parts (split form).
template <int SPLIT>
__device__ __forceinline__ void hpass(const __half *pl, int hb, int warp, const unsigned (&ah)[2][4],
                                      const unsigned (&al)[2][4], unsigned (&hh)[4][2][2], unsigned (&hl)[4][2][2]) {
    using G = SsimMmaGeom<SPLIT>;
    const int lane = threadIdx.x & 31;
    const int off = (16 * hb + (lane & 7)) * MT_LD + 16 * warp + 8 * (lane >> 3);
#pragma unroll
    for (int p = 0; p < 4; p++) {
#pragma unroll
        for (int nt = 0; nt < 2; nt++) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            unsigned b[4];
            ldmatrix_x4(b, pl + p * G::PLANE + off + 8 * nt * MT_LD);
            if (SPLIT != 1) {
                unsigned bl[4];
                ldmatrix_x4(bl, pl + (p + 4) * G::PLANE + off + 8 * nt * MT_LD);
                // small products first
                iqm::mma_f16_16816(acc, al[0], b[0], b[1]);
                iqm::mma_f16_16816(acc, al[1], b[2], b[3]);
                iqm::mma_f16_16816(acc, ah[0], bl[0], bl[1]);
                iqm::mma_f16_16816(acc, ah[1], bl[2], bl[3]);
            }
            iqm::mma_f16_16816(acc, ah[0], b[0], b[1]);
            iqm::mma_f16_16816(acc, ah[1], b[2], b[3]);
            // acc: (output column g / g + 8, block rows 8 nt + 2t, 2t + 1)
            if (SPLIT == 1) {
                hh[p][0][nt] = iqm::pack_h2(acc[0], acc[1]);
                hh[p][1][nt] = iqm::pack_h2(acc[2], acc[3]);
            } else {
                iqm::split_h2(acc[0], acc[1], hh[p][0][nt], hl[p][0][nt]);
                iqm::split_h2(acc[2], acc[3], hh[p][1][nt], hl[p][1][nt]);
            }
        }
    }
}

// Vertical block: out[p][v][i] for output rows g (i < 2) / g + 8 (i >= 2), columns 8v + 2t + (i & 1),
// from the horizontal blocks above (h0: k rows 0-15 of the window) and below (h1: k rows 16-31).
template <int SPLIT>
__device__ __forceinline__ void vpass(const unsigned (&ah)[2][4], const unsigned (&al)[2][4],
                                      const unsigned (&h0h)[4][2][2], const unsigned (&h0l)[4][2][2],
                                      const unsigned (&h1h)[4][2][2], const unsigned (&h1l)[4][2][2],
                                      float (&out)[4][2][4]) {
#pragma unroll
    for (int p = 0; p < 4; p++) {
#pragma unroll
        for (int v = 0; v < 2; v++) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            if (SPLIT != 1) {
                iqm::mma_f16_16816(acc, al[0], h0h[p][v][0], h0h[p][v][1]);
                iqm::mma_f16_16816(acc, al[1], h1h[p][v][0], h1h[p][v][1]);
                iqm::mma_f16_16816(acc, ah[0], h0l[p][v][0], h0l[p][v][1]);
                iqm::mma_f16_16816(acc, ah[1], h1l[p][v][0], h1l[p][v][1]);
            }
            iqm::mma_f16_16816(acc, ah[0], h0h[p][v][0], h0h[p][v][1]);
            iqm::mma_f16_16816(acc, ah[1], h1h[p][v][0], h1h[p][v][1]);
#pragma unroll
            for (int i = 0; i < 4; i++) out[p][v][i] = acc[i];
        }
    }
}

// The pair of a work unit (pairs sorted by unit_base).
__device__ __forceinline__ int find_unit(const SsimPairDev *pairs, int n, int unit) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (pairs[mid].unit_base <= unit) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// In-image sum of the effective window taps around position x of a line of length n.
__device__ __forceinline__ float window_sum(const float *w, int R, int x, int n) {
    float s = 0.f;
    for (int k = 0; k <= 2 * R; k++) {
        const int xx = x + k - R;
        s += (xx >= 0 && xx < n) ? w[k] : 0.f;
    }
    return s;
}

// SSIM of one output pixel from its four window sums (m1: shifted first moments of u, v; m2: second
// moments), `inv` the normalisation (1 / (window weight * 2^12)), (cu, cv) the tile's shift.
__device__ __forceinline__ float ssim_px(float2 m1, float2 m2, float inv, float cu, float cv, float c1, float c2) {
    const float2 iv = make_float2(inv, inv);
    const float2 sm = __fmul2_rn(m1, iv);                                     // shifted means
    const float2 var = __ffma2_rn(m2, iv, __fmul2_rn(sm, make_float2(-sm.x, -sm.y)));
    const float2 mu = __fadd2_rn(sm, make_float2(cu, cv));
    const float2 mu2 = __fmul2_rn(mu, mu);
    // (mean term, variance term) of u and of v; SSIM = prod(0.5 (X - Y) + C) / prod(0.5 (X + Y) + C)
    const float2 X = make_float2(mu2.x, var.x), Y = make_float2(mu2.y, var.y), C = make_float2(c1, c2);
    const float2 plus = __ffma2_rn(__fadd2_rn(X, Y), make_float2(0.5f, 0.5f), C);
    const float2 minus = __ffma2_rn(__ffma2_rn(Y, make_float2(-1.f, -1.f), X), make_float2(0.5f, 0.5f), C);
    return (minus.x * minus.y) * iqm::rcp_approx(plus.x * plus.y);  // plus.x plus.y >= c1 c2 > 0
}

// Persistent: each CTA walks tiles blockIdx.x, blockIdx.x + gridDim.x, ... (neighbouring tiles run
// at the same time, so the rows they share meet in L2), keeping the band fragments and a warm
// instruction cache across tiles.
template <int SPLIT>
__global__ void __launch_bounds__(MT_THREADS, SPLIT == 1 ? MT_MIN_CTAS_SINGLE : MT_MIN_CTAS_SPLIT) ssim_mma_kernel(SsimMmaArgs args, int total_units) {
    extern __shared__ __align__(16) unsigned char ssim_mma_smem[];
    __half *pl = reinterpret_cast<__half *>(ssim_mma_smem);
    __shared__ double red[MT_THREADS / 32];
    __shared__ int is_last;
    __shared__ float gsh[16];   // the normalised taps g(-R..R), zero beyond
    __shared__ float weff[16];  // the taps as the tensor cores apply them

    const int R = args.R;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;

    // the taps into shared memory (a kernel-parameter array indexed at run time would be copied
    // to local memory whole): gsh as given, weff as the tensor cores apply them
    if (threadIdx.x < 16) {
        float v = 0.f;
#pragma unroll
        for (int k = 0; k < 15; k++)
            if (int(threadIdx.x) == k) v = args.gn[k];
        float w = __half2float(__float2half_rn(v));
        if (SPLIT != 1) w += __half2float(__float2half_rn(v - w));
        gsh[threadIdx.x] = v;
        weff[threadIdx.x] = w;
    }
    __syncthreads();

    // band fragments: Gb[m][j] = gn[j - 8 - m + R] where that index lies in 0..2R
    unsigned ah[2][4], al[2][4];
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int m = g + 8 * (i & 1);
            const int j = 16 * s + 2 * t + 8 * (i >> 1);
            const int k0 = j - 8 - m + R, k1 = k0 + 1;
            const float v0 = (k0 >= 0 && k0 <= 2 * R) ? gsh[k0] : 0.f;
            const float v1 = (k1 >= 0 && k1 <= 2 * R) ? gsh[k1] : 0.f;
            if (SPLIT == 1) {
                ah[s][i] = iqm::pack_h2(v0, v1);
                al[s][i] = 0u;
            } else {
                iqm::split_h2(v0, v1, ah[s][i], al[s][i]);
            }
        }
    float wsum = 0.f;  // interior window sum (1 up to the taps' rounding)
    for (int k = 0; k <= 2 * R; k++) wsum += weff[k];
    const float inv_in = 1.0f / (wsum * wsum * MT_SCALE);

    // A work unit is a column segment of SEGT vertically adjacent tiles of one pair, walked top to
    // bottom.  The split form uses one shift for the segment, so each tile after the first takes its
    // first horizontal block (image rows y0 - 8 .. y0 + 7) from the previous tile's last one, still
    // in registers, and stages only the 64 rows below it.  The single-product form keeps one shift
    // per tile (its error grows with the shift tile) and stages every tile whole.
    constexpr int SEGT = MT_SEG_SPLIT;
    constexpr bool SHARE = SPLIT != 1;  // one shift per segment, the boundary block reused
    unsigned hph[4][2][2], hpl[4][2][2], hnh[4][2][2], hnl[4][2][2];
    for (int unit = blockIdx.x; unit < total_units; unit += gridDim.x) {
        const int pi = find_unit(args.pairs, args.npairs, unit);
        const SsimPairDev P = args.pairs[pi];
        const int W = P.w, H = P.h;
        const int local = unit - P.unit_base;
        const int tx = local % P.tiles_x, ty0 = (local / P.tiles_x) * SEGT;
        const int ty1 = min(ty0 + SEGT, P.ntiles / P.tiles_x);
        const int x0 = tx * MT_W;

        // shift constants: u, v of the segment's (SHARE) or the tile's centre pixel
        float cu = 0.f, cv = 0.f;
        auto shift_at = [&](int cy) {
            const int cx = min(x0 + MT_W / 2, W - 1);
            cy = min(cy, H - 1);
            const uint32_t pa = __ldg(reinterpret_cast<const uint32_t *>(P.a + (long long)cy * P.pitch) + cx);
            const uint32_t pb = __ldg(reinterpret_cast<const uint32_t *>(P.b + (long long)cy * P.pitch) + cx);
            const float2 l = luma2(pa, pb);
            cu = l.x + l.y;
            cv = l.x - l.y;
        };
        if (SHARE) shift_at((ty0 + ty1) * MT_H / 2);

        // normalisation of the lane's columns (2t, 2t + 1 of each 8-column half): the window weight
        // cut at the image border, relative to the interior one
        const bool interior_x = x0 >= R && x0 + MT_W - 1 + R <= W - 1;
        float rx[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int x = x0 + 16 * warp + 8 * (j >> 1) + 2 * t + (j & 1);
            rx[j] = interior_x ? 1.f : wsum / window_sum(weff, R, x, W);
        }

#pragma unroll 1
        for (int ty = ty0; ty < ty1; ty++) {
            const int y0 = ty * MT_H;
            const int hb0 = SHARE && ty != ty0 ? 1 : 0;  // first horizontal block computed here
            if (!SHARE) shift_at(y0 + MT_H / 2);

            // the previous tile's ldmatrix reads ended before the barriers of its pooling
            stage_moments<SPLIT>(pl, P, x0, y0, cu, cv, 16 * hb0);
            __syncthreads();

            // every output pixel in the image, under the full window and pooled
            const bool interior = interior_x && y0 >= R && y0 + MT_H - 1 + R <= H - 1;

            float acc = 0.f;
#pragma unroll 1
            for (int hb = hb0; hb < MT_ROWS / 16; hb++) {
                hpass<SPLIT>(pl, hb, warp, ah, al, hnh, hnl);
                if (hb > 0) {
                    // output rows y0 + 16 (hb - 1) + 0..15 from the window of blocks hb - 1 and hb
                    float out[4][2][4];
                    vpass<SPLIT>(ah, al, hph, hpl, hnh, hnl, out);
                    const int yb = y0 + 16 * (hb - 1) + g;
                    float ry[2];  // 1 / (window weight * 2^12) of the lane's rows g, g + 8
#pragma unroll
                    for (int e = 0; e < 2; e++)
                        ry[e] = interior ? inv_in : inv_in * wsum / window_sum(weff, R, yb + 8 * e, H);
#pragma unroll
                    for (int i = 0; i < 4; i++)
#pragma unroll
                        for (int v = 0; v < 2; v++) {
                            const int y = yb + 8 * (i >> 1);
                            const int x = x0 + 16 * warp + 8 * v + 2 * t + (i & 1);
                            const float ssim = ssim_px(make_float2(out[0][v][i], out[1][v][i]),
                                                       make_float2(out[2][v][i], out[3][v][i]),
                                                       ry[i >> 1] * rx[2 * v + (i & 1)], cu, cv, args.c1, args.c2);
                            const bool valid = interior || (x < W && y < H);
                            if (valid && P.map) P.map[(long long)y * W + x] = ssim;
                            const bool pool = interior || (valid && x >= R && x <= W - R && y >= R && y <= H - R);
                            acc += pool ? ssim : 0.f;
                        }
                }
#pragma unroll
                for (int p = 0; p < 4; p++)
#pragma unroll
                    for (int v = 0; v < 2; v++)
#pragma unroll
                        for (int kb = 0; kb < 2; kb++) {
                            hph[p][v][kb] = hnh[p][v][kb];
                            hpl[p][v][kb] = hnl[p][v][kb];
                        }
            }

            pool_tiles<MT_THREADS>(acc, red, &is_last, args.partials, args.counters, args.scores, pi, P,
                                   P.tile_base + ty * P.tiles_x + tx, double(W - 2 * R + 1) * double(H - 2 * R + 1));
        }
    }
}

}  // namespace
