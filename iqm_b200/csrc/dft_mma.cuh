// Warp-level DFT on the tensor cores (mma.sync m16n8k16, FP16 operands, FP32 accumulation).
//
// A transform of length N = N1 * N2 (N1 <= 16, N2 <= 32) is computed as two dense DFT stages with a
// twiddle between them (the two-factor Cooley-Tukey split, n = N2 n1 + n2, k = k1 + N1 k2):
//   Y[k1][n2] = sum_n1 x[N2 n1 + n2] w_N1^(k1 n1)          stage A: DFT-N1 over n1, batch n2
//   Y[k1][n2] *= w_N^(k1 n2)                                 twiddle
//   X[k1 + N1 k2] = sum_n2 Y[k1][n2] w_N2^(n2 k2)             stage C: DFT-N2 over n2, batch k1
// with w_L = exp(sign 2 pi i / L).  Complex products run as real matrix products:
//   stage A: the DFT-N1 matrix in real form is the A operand (rows 0-15: Re of output k1, rows
//            16-31: Im; columns 2 n1 + c: Re / Im of input n1), the data the B operand (columns n2);
//   stage C: stage A's accumulators, twiddled and rounded to FP16, are the A operand as they stand
//            (rows k1; columns: Re of n2 for the first 8 NT2 columns, then Im) -- the C fragment of
//            two m16n8 tiles is exactly the A fragment of one m16n8k16 tile, so the data never
//            leaves registers between the stages -- and the DFT-N2 matrix in real form the B operand
//            (columns 2 k2 + c: Re / Im of output k2).
// Each lane (g = lane / 4, t = lane % 4) reads its share of the input (12 points at 270 = 15 x 18,
// 16 at 480 = 16 x 30) and ends with its share of the output as complex pairs.  The constants are
// built once into a global table (build); each CTA copies the stage-C matrix and the twiddles, the
// same for every warp, into one lane-indexed shared-memory table (conflict-free 8-byte loads) and
// keeps only the stage-A matrix in registers, which leaves room for several CTAs per SM.
//
// SPLIT = 3 adds the split-precision products: operands as hi + lo FP16 pairs (hi = fp16(v),
// lo = fp16(v - hi)) and A B ~ A_hi B_hi + A_hi B_lo + A_lo B_hi, about 21 significant bits per
// product instead of 11.  SPLIT = 1 uses the hi parts alone.
//
// Operand ranges: FP16 holds magnitudes up to 65504, so callers scale inputs (the FSIM passes
// divide by the plane size N first, which keeps every value of the normalised transforms in range).
#pragma once

#include <cuda_fp16.h>

#include <type_traits>

namespace iqm {

__device__ __forceinline__ void mma_f16_16816(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ unsigned h2_bits(__half2 h) { return *reinterpret_cast<unsigned *>(&h); }

// (x, y) as an FP16 pair, x in the low half (the lower matrix index of a fragment register).
__device__ __forceinline__ unsigned pack_h2(float x, float y) { return h2_bits(__floats2half2_rn(x, y)); }

// hi = fp16(x, y), lo = fp16((x, y) - hi)
__device__ __forceinline__ void split_h2(float x, float y, unsigned &hi, unsigned &lo) {
    const __half2 h = __floats2half2_rn(x, y);
    const float2 hf = __half22float2(h);
    hi = h2_bits(h);
    lo = h2_bits(__floats2half2_rn(x - hf.x, y - hf.y));
}

// exp(sign 2 pi i m / L) for 0 <= m < L, from the exactly reduced angle
__device__ __forceinline__ float2 unit_root(int m, int L, float sign) {
    float s, c;
    sincospif(2.0f * float(m) / float(L), &s, &c);
    return make_float2(c, sign * s);
}

// REGS: keep the stage-C matrix and the twiddles in registers instead of the shared table (fewer
// shared-memory loads per transform, more registers).
template <int N1_, int N2_, int SPLIT, bool REGS = false>
struct MmaDft {
    static constexpr int N1 = N1_, N2 = N2_, N = N1 * N2;
    static constexpr int NT2 = (N2 + 7) / 8;      // stage A column tiles (n2); stage C k-tiles
    static constexpr int NTC = (2 * N2 + 7) / 8;  // stage C column tiles (2 k2 + c)
    static constexpr int P = SPLIT == 1 ? 1 : 2;  // parts of each constant (hi, lo)
    static constexpr bool kRegs = REGS;
    static_assert(N1 >= 2 && N1 <= 16 && N2 >= 2 && N2 <= 32, "factor range of the MMA engine");
    static_assert(SPLIT == 1 || SPLIT == 3, "SPLIT is 1 or 3 products");

    // Tables: the stage-A fragments of every lane, [part][m-tile][k-tile][register][lane] as 32-bit
    // words, then the stage-C matrix [part][k-tile][n-tile][lane] as register pairs, then the
    // twiddle of (k1 = g + 8 r, n2 = 8 j + 2 t + e) as [r][j][e][lane].  build() writes the whole
    // table to global memory once; load() copies the stage-C and twiddle parts into the CTA's shared
    // memory and the lane's stage-A fragments into registers.
    static constexpr int FA_WORDS = P * 2 * 2 * 4 * 32;
    static constexpr int FC_ENTRIES = P * NT2 * NTC * 32;
    static constexpr int TW_ENTRIES = 2 * NT2 * 2 * 32;
    static constexpr size_t shared_part = sizeof(uint2) * FC_ENTRIES + sizeof(float2) * TW_ENTRIES;
    static constexpr size_t smem_bytes = REGS ? 0 : shared_part;  // shared memory the engine needs
    static constexpr size_t table_bytes = sizeof(unsigned) * FA_WORDS + shared_part;
    static_assert(sizeof(unsigned) * FA_WORDS % 16 == 0 && shared_part % 16 == 0, "16-byte table parts");

    unsigned fa[P][2][2][4];  // stage A matrix: [part][m-tile: Re/Im out][k-tile][register]
    const uint2 *fcs;         // shared stage C table
    const float2 *tws;        // shared twiddle table
    uint2 fcr[REGS ? P : 1][REGS ? NT2 : 1][REGS ? NTC : 1];  // the same in registers (REGS)
    float2 twr[REGS ? 2 : 1][REGS ? NT2 : 1][REGS ? 2 : 1];

    __device__ __forceinline__ uint2 fc_at(int p, int kc, int nc) const {
        if constexpr (REGS) {
            return fcr[p][kc][nc];
        } else {
            return fcs[((p * NT2 + kc) * NTC + nc) * 32 + (threadIdx.x & 31)];
        }
    }
    __device__ __forceinline__ float2 tw_at(int r, int j, int e) const {
        if constexpr (REGS) {
            return twr[r][j][e];
        } else {
            return tws[((r * NT2 + j) * 2 + e) * 32 + (threadIdx.x & 31)];
        }
    }

    // Writes the table for transforms of sign `sign` (+1 inverse, -1 forward); run by one warp.
    static __device__ void build(void *table, float sign) {
        const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
        unsigned *fa_w = static_cast<unsigned *>(table);
        uint2 *fc_w = reinterpret_cast<uint2 *>(fa_w + FA_WORDS);
        float2 *tw_w = reinterpret_cast<float2 *>(fc_w + FC_ENTRIES);
        auto put = [&](unsigned *hi, unsigned *lo, float x, float y) {
            if constexpr (SPLIT == 1) {
                *hi = pack_h2(x, y);
            } else {
                split_h2(x, y, *hi, *lo);
            }
        };
        for (int mt = 0; mt < 2; mt++)
            for (int kt = 0; kt < 2; kt++)
                for (int q = 0; q < 4; q++) {
                    // register q: rows g (q even) / g + 8 (q odd); columns 2 t, 2 t + 1 (+ 8 for q >= 2)
                    const int k1 = g + 8 * (q & 1);
                    const int n1 = 8 * kt + t + 4 * (q >> 1);
                    float vr = 0.f, vi = 0.f;  // coefficients of input Re and input Im
                    if (k1 < N1 && n1 < N1) {
                        const float2 w = unit_root((k1 * n1) % N1, N1, sign);
                        vr = mt == 0 ? w.x : w.y;
                        vi = mt == 0 ? -w.y : w.x;
                    }
                    unsigned hi, lo;
                    put(&hi, &lo, vr, vi);
                    fa_w[(((0 * 2 + mt) * 2 + kt) * 4 + q) * 32 + lane] = hi;
                    if constexpr (P == 2) fa_w[(((1 * 2 + mt) * 2 + kt) * 4 + q) * 32 + lane] = lo;
                }
        for (int kc = 0; kc < NT2; kc++)
            for (int nc = 0; nc < NTC; nc++) {
                unsigned hi[2], lo[2];
                for (int q = 0; q < 2; q++) {
                    // rows 16 kc + 8 q + 2 t + {0, 1} (half-tile h = 2 kc + q: Re / Im block c, n2),
                    // column 8 nc + g (output k2 = (8 nc + g) / 2, Re / Im part cc)
                    const int h = 2 * kc + q;
                    const int c = h / NT2, n2 = 8 * (h % NT2) + 2 * t;
                    const int k2 = (8 * nc + g) >> 1, cc = g & 1;
                    float v[2];
                    for (int e = 0; e < 2; e++) {
                        v[e] = 0.f;
                        if (n2 + e < N2 && k2 < N2) {
                            const float2 w = unit_root(((n2 + e) * k2) % N2, N2, sign);
                            // Re out: Yr wr - Yi wi ; Im out: Yr wi + Yi wr
                            v[e] = c == 0 ? (cc == 0 ? w.x : w.y) : (cc == 0 ? -w.y : w.x);
                        }
                    }
                    put(&hi[q], &lo[q], v[0], v[1]);
                }
                fc_w[(kc * NTC + nc) * 32 + lane] = make_uint2(hi[0], hi[1]);
                if constexpr (P == 2) fc_w[((NT2 + kc) * NTC + nc) * 32 + lane] = make_uint2(lo[0], lo[1]);
            }
        for (int r = 0; r < 2; r++)
            for (int j = 0; j < NT2; j++)
                for (int e = 0; e < 2; e++) {
                    const int k1 = g + 8 * r, n2 = 8 * j + 2 * t + e;
                    tw_w[((r * NT2 + j) * 2 + e) * 32 + lane] = unit_root((k1 * n2) % N, N, sign);
                }
    }

    // Copies the shared part of `table` (global, from build) into `shared` (smem_bytes, 16-byte
    // aligned) with every thread of the CTA, and this lane's stage-A fragments into registers.  The
    // caller synchronises the CTA before the first run().
    __device__ __forceinline__ void load(const void *table, void *shared) {
        const int lane = threadIdx.x & 31;
        const unsigned *fa_g = static_cast<const unsigned *>(table);
#pragma unroll
        for (int p = 0; p < P; p++)
#pragma unroll
            for (int mt = 0; mt < 2; mt++)
#pragma unroll
                for (int kt = 0; kt < 2; kt++)
#pragma unroll
                    for (int q = 0; q < 4; q++) fa[p][mt][kt][q] = __ldg(fa_g + (((p * 2 + mt) * 2 + kt) * 4 + q) * 32 + lane);
        if constexpr (REGS) {
            const uint2 *fc_g = reinterpret_cast<const uint2 *>(fa_g + FA_WORDS);
            const float2 *tw_g = reinterpret_cast<const float2 *>(fc_g + FC_ENTRIES);
#pragma unroll
            for (int p = 0; p < P; p++)
#pragma unroll
                for (int kc = 0; kc < NT2; kc++)
#pragma unroll
                    for (int nc = 0; nc < NTC; nc++) fcr[p][kc][nc] = __ldg(fc_g + ((p * NT2 + kc) * NTC + nc) * 32 + lane);
#pragma unroll
            for (int r = 0; r < 2; r++)
#pragma unroll
                for (int j = 0; j < NT2; j++)
#pragma unroll
                    for (int e = 0; e < 2; e++) twr[r][j][e] = __ldg(tw_g + ((r * NT2 + j) * 2 + e) * 32 + lane);
            (void)shared;
        } else {
            const uint4 *src = reinterpret_cast<const uint4 *>(fa_g + FA_WORDS);
            uint4 *dst = static_cast<uint4 *>(shared);
            for (int i = threadIdx.x; i < int(smem_bytes / 16); i += blockDim.x) dst[i] = __ldg(src + i);
            fcs = static_cast<const uint2 *>(shared);
            tws = reinterpret_cast<const float2 *>(fcs + FC_ENTRIES);
        }
    }

    // Output slot s of a lane (0 <= s < 2 NTC) holds X[k1 + N1 k2] with k1 = g + 8 (s & 1),
    // k2 = 4 (s >> 1) + t when both are in range.
    static __device__ __forceinline__ int slot_k1(int s) { return ((threadIdx.x & 31) >> 2) + 8 * (s & 1); }
    static __device__ __forceinline__ int slot_k2(int s) { return 4 * (s >> 1) + (threadIdx.x & 3); }

    // One transform.  ld(n1, n2) returns the (already scaled) input x[N2 n1 + n2] for n1 < N1,
    // n2 < N2, either as float2 or, for inputs that already are FP16, as the raw bits of a __half2
    // (real part in the low half), which go into the MMA operand as they are (and, being exact,
    // need no lo part in the split form); st(k, slot, v) receives output X[k] (in this lane's
    // `slot`) for every k < N exactly once across the warp.  All 32 lanes must call it together
    // (warp-synchronous MMAs).
    template <class Load, class Store>
    __device__ __forceinline__ void run(Load ld, Store st) const {
        const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
        float acc[2][NT2][4];
#pragma unroll
        for (int mt = 0; mt < 2; mt++)
#pragma unroll
            for (int j = 0; j < NT2; j++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[mt][j][q] = 0.f;
        // stage A
#pragma unroll
        for (int j = 0; j < NT2; j++) {
            const int n2 = 8 * j + g;
#pragma unroll
            for (int kt = 0; kt < 2; kt++) {
                const int n1a = 8 * kt + t, n1b = n1a + 4;
                if constexpr (std::is_same<decltype(ld(0, 0)), unsigned>::value) {
                    const unsigned b0 = (n1a < N1 && n2 < N2) ? ld(n1a, n2) : 0u;
                    const unsigned b1 = (n1b < N1 && n2 < N2) ? ld(n1b, n2) : 0u;
#pragma unroll
                    for (int mt = 0; mt < 2; mt++) {
                        mma_f16_16816(acc[mt][j], fa[0][mt][kt], b0, b1);
                        if constexpr (SPLIT == 3) mma_f16_16816(acc[mt][j], fa[1][mt][kt], b0, b1);
                    }
                } else {
                    const float2 xa = (n1a < N1 && n2 < N2) ? ld(n1a, n2) : make_float2(0.f, 0.f);
                    const float2 xb = (n1b < N1 && n2 < N2) ? ld(n1b, n2) : make_float2(0.f, 0.f);
                    if constexpr (SPLIT == 1) {
                        const unsigned b0 = pack_h2(xa.x, xa.y), b1 = pack_h2(xb.x, xb.y);
#pragma unroll
                        for (int mt = 0; mt < 2; mt++) mma_f16_16816(acc[mt][j], fa[0][mt][kt], b0, b1);
                    } else {
                        unsigned h0, l0, h1, l1;
                        split_h2(xa.x, xa.y, h0, l0);
                        split_h2(xb.x, xb.y, h1, l1);
#pragma unroll
                        for (int mt = 0; mt < 2; mt++) {
                            mma_f16_16816(acc[mt][j], fa[0][mt][kt], h0, h1);
                            mma_f16_16816(acc[mt][j], fa[0][mt][kt], l0, l1);
                            mma_f16_16816(acc[mt][j], fa[1][mt][kt], h0, h1);
                        }
                    }
                }
            }
        }
        // twiddle: registers 0, 1 hold row g (k1 = g), 2, 3 row g + 8; even / odd: n2 = 8 j + 2 t + e
#pragma unroll
        for (int j = 0; j < NT2; j++)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float2 w = tw_at(q >> 1, j, q & 1);
                const float re = acc[0][j][q], im = acc[1][j][q];
                acc[0][j][q] = re * w.x - im * w.y;
                acc[1][j][q] = re * w.y + im * w.x;
            }
        // stage C: k-tile kc is made of half-tiles 2 kc and 2 kc + 1 (half h: block c = h / NT2,
        // n2 tile j = h % NT2), each one m16n8 accumulator tile of stage A
        float out[NTC][4];
#pragma unroll
        for (int nc = 0; nc < NTC; nc++)
#pragma unroll
            for (int q = 0; q < 4; q++) out[nc][q] = 0.f;
#pragma unroll
        for (int kc = 0; kc < NT2; kc++) {
            const int h0 = 2 * kc, h1 = 2 * kc + 1;
            const float *c0 = acc[h0 / NT2][h0 % NT2];
            const float *c1 = acc[h1 / NT2][h1 % NT2];
            if constexpr (SPLIT == 1) {
                const unsigned a[4] = {pack_h2(c0[0], c0[1]), pack_h2(c0[2], c0[3]), pack_h2(c1[0], c1[1]),
                                       pack_h2(c1[2], c1[3])};
#pragma unroll
                for (int nc = 0; nc < NTC; nc++) {
                    const uint2 b = fc_at(0, kc, nc);
                    mma_f16_16816(out[nc], a, b.x, b.y);
                }
            } else {
                unsigned ah[4], al[4];
                split_h2(c0[0], c0[1], ah[0], al[0]);
                split_h2(c0[2], c0[3], ah[1], al[1]);
                split_h2(c1[0], c1[1], ah[2], al[2]);
                split_h2(c1[2], c1[3], ah[3], al[3]);
#pragma unroll
                for (int nc = 0; nc < NTC; nc++) {
                    const uint2 bh = fc_at(0, kc, nc);
                    const uint2 bl = fc_at(1, kc, nc);
                    mma_f16_16816(out[nc], ah, bh.x, bh.y);
                    mma_f16_16816(out[nc], al, bh.x, bh.y);
                    mma_f16_16816(out[nc], ah, bl.x, bl.y);
                }
            }
        }
        // outputs: tile nc, registers (0, 1) = (Re, Im) of X[k1 = g][k2 = 4 nc + t], (2, 3) of k1 = g + 8
#pragma unroll
        for (int nc = 0; nc < NTC; nc++) {
            const int k2 = 4 * nc + t;
            if (k2 < N2) {
                if (g < N1) st(g + N1 * k2, 2 * nc, make_float2(out[nc][0], out[nc][1]));
                if (g + 8 < N1) st(g + 8 + N1 * k2, 2 * nc + 1, make_float2(out[nc][2], out[nc][3]));
            }
        }
    }
};

}  // namespace iqm
