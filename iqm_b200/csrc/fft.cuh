// Complex FP32 FFTs in shared memory (sm_100a), the transform engine behind FSIM.
//
// The reference delegates its FFTs to VkFFT (src/gpu/fsim/fsim.cpp:201-263 plans, :364 forward
// with sign -1 and no scaling, :378 inverse with sign +1 and normalize = 1/N).  Here a transform
// of length n runs inside one CTA as a Stockham auto-sort FFT: log_p stages, each reading one
// buffer and writing the other, so no bit reversal is needed.  n is factored into radices
// computed in registers (2, 3, 4, 5, 6, 8, 9, 10, 12, 15) and other odd primes up to 251 (a direct
// O(p^2) butterfly, read from the length's table); when that is estimated dearer, or a prime factor
// is larger, the length runs through Bluestein's chirp-z algorithm on the smallest 2,3,5-smooth
// length m >= 2n-1.
//
// Stage s with radix p and stride L (the product of the earlier radices), butterfly j in [0, n/p):
//   k = j mod L;  v_r = in[j + r n/p] * W^(r k),  W = exp(sign 2 pi i / (L p));
//   V = DFT_p(v);  out[(j / L) L p + k + q L] = V_q.
// Twiddles come from a per-length table exp(-2 pi i t / n), t < n, evaluated in double on the host
// and rounded to float (conjugated for sign = +1).
#pragma once

#include <cuda_runtime.h>

namespace iqm {

constexpr int FFT_MAX_STAGES = 16;
constexpr int FFT_MAX_GENERIC = 251;  // largest prime the planner may give a direct butterfly

// Device-visible description of one transform length.
struct FftLen {
    int n;
    int nst;
    int radix[FFT_MAX_STAGES];
    int stride[FFT_MAX_STAGES];    // L: product of the earlier radices
    float inv_stride[FFT_MAX_STAGES];
    float inv_q[FFT_MAX_STAGES];   // 1 / (n / radix)
    int stw_off[FFT_MAX_STAGES];   // offset of each stage's twiddles in stw
    int stw_len;                   // entries of stw: sum over stages of (radix - 1) * stride
    const float2 *stw;        // stage twiddles W_{L p}^{r k} (sign -1), [k][r-1] per stage
    const float2 *tw;         // n entries, exp(-2 pi i t / n)
    // Bluestein data (bluestein != 0): x -> c * IFFT_m( FFT_m(c * x) * B ), c = chirp
    int bluestein;
    int m;
    int mst;
    int mradix[FFT_MAX_STAGES];
    int mstride[FFT_MAX_STAGES];
    float minv_stride[FFT_MAX_STAGES];
    float minv_q[FFT_MAX_STAGES];
    int mstw_off[FFT_MAX_STAGES];
    int mstw_len;
    const float2 *mstw;
    const float2 *mtw;        // m entries, exp(-2 pi i t / m)
    const float2 *chirp;      // n entries, exp(-pi i t^2 / n)
    const float2 *bfwd;       // m entries, FFT_m(conj chirp, wrapped) / m      (sign -1)
    const float2 *binv;       // m entries, FFT_m(chirp, wrapped) / m           (sign +1)
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// complex sum and difference as one packed FP32x2 add each (both halves rounded like scalar adds)
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
// multiply by i*s (s = +-1)
__device__ __forceinline__ float2 cmul_is(float2 a, float s) { return make_float2(-s * a.y, s * a.x); }
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }

__device__ __forceinline__ float2 tw_at(const float2 *tw, int idx, float s) {
    const float2 w = __ldg(tw + idx);
    return make_float2(w.x, -s * w.y);  // table holds sign -1; s = sign
}

// DFT of p points in registers, sign s: V_q = sum_r v_r exp(s 2 pi i r q / p).
template <int P>
__device__ __forceinline__ void dft_small(float2 *v, float s);

template <>
__device__ __forceinline__ void dft_small<2>(float2 *v, float s) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}
template <>
__device__ __forceinline__ void dft_small<3>(float2 *v, float s) {
    const float c = 0.86602540378443865f;  // sqrt(3)/2
    const float2 t1 = cadd(v[1], v[2]);
    const float2 t2 = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
    const float2 d = csub(v[1], v[2]);
    const float2 t3 = cmul_is(make_float2(c * d.x, c * d.y), s);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
}
template <>
__device__ __forceinline__ void dft_small<4>(float2 *v, float s) {
    const float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    const float2 b0 = cadd(v[1], v[3]), b1 = cmul_is(csub(v[1], v[3]), s);
    v[0] = cadd(a0, b0);
    v[2] = csub(a0, b0);
    v[1] = cadd(a1, b1);
    v[3] = csub(a1, b1);
}
template <>
__device__ __forceinline__ void dft_small<5>(float2 *v, float s) {
    const float c1 = 0.30901699437494742f, c2 = -0.80901699437494742f;
    const float s1 = 0.95105651629515357f, s2 = 0.58778525229247313f;
    const float2 p14 = cadd(v[1], v[4]), m14 = csub(v[1], v[4]);
    const float2 p23 = cadd(v[2], v[3]), m23 = csub(v[2], v[3]);
    const float2 a0 = v[0];
    const float2 r1 = make_float2(a0.x + c1 * p14.x + c2 * p23.x, a0.y + c1 * p14.y + c2 * p23.y);
    const float2 r2 = make_float2(a0.x + c2 * p14.x + c1 * p23.x, a0.y + c2 * p14.y + c1 * p23.y);
    const float2 i1 = cmul_is(make_float2(s1 * m14.x + s2 * m23.x, s1 * m14.y + s2 * m23.y), s);
    const float2 i2 = cmul_is(make_float2(s2 * m14.x - s1 * m23.x, s2 * m14.y - s1 * m23.y), s);
    v[0] = cadd(a0, cadd(p14, p23));
    v[1] = cadd(r1, i1);
    v[4] = csub(r1, i1);
    v[2] = cadd(r2, i2);
    v[3] = csub(r2, i2);
}
template <>
__device__ __forceinline__ void dft_small<8>(float2 *v, float s) {
    float2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    dft_small<4>(e, s);
    dft_small<4>(o, s);
    const float h = 0.70710678118654752f;
    // W8^q for q = 0..3 with W8 = exp(s 2 pi i / 8)
    const float2 w1 = make_float2(h, s * h), w3 = make_float2(-h, s * h);
    const float2 t0 = o[0];
    const float2 t1 = cmul(o[1], w1);
    const float2 t2 = cmul_is(o[2], s);
    const float2 t3 = cmul(o[3], w3);
    v[0] = cadd(e[0], t0); v[4] = csub(e[0], t0);
    v[1] = cadd(e[1], t1); v[5] = csub(e[1], t1);
    v[2] = cadd(e[2], t2); v[6] = csub(e[2], t2);
    v[3] = cadd(e[3], t3); v[7] = csub(e[3], t3);
}

// Composite sizes from the small kernels above.  Coprime N1 x N2 (6, 10, 12, 15): Good-Thomas
// prime-factor mapping, input n = (N2 n1 + N1 n2) mod N, output k = (N2 a k1 + N1 b k2) mod N with
// a = N2^-1 mod N1 and b = N1^-1 mod N2, so no twiddles are needed between the two passes.
__host__ __device__ constexpr int mod_inverse(int x, int m) {
    for (int i = 1; i < m; i++)
        if ((x * i) % m == 1) return i;
    return 1;
}

template <int N1, int N2>
__device__ __forceinline__ void dft_pfa(float2 *v, float s) {
    constexpr int N = N1 * N2;
    constexpr int A = mod_inverse(N2 % N1, N1), B = mod_inverse(N1 % N2, N2);
    float2 t[N2][N1];
#pragma unroll
    for (int n2 = 0; n2 < N2; n2++) {
        float2 a[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; n1++) a[n1] = v[(n1 * N2 + n2 * N1) % N];
        dft_small<N1>(a, s);
#pragma unroll
        for (int k1 = 0; k1 < N1; k1++) t[n2][k1] = a[k1];
    }
#pragma unroll
    for (int k1 = 0; k1 < N1; k1++) {
        float2 b[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; n2++) b[n2] = t[n2][k1];
        dft_small<N2>(b, s);
#pragma unroll
        for (int k2 = 0; k2 < N2; k2++) v[(k1 * N2 * A + k2 * N1 * B) % N] = b[k2];
    }
}

template <>
__device__ __forceinline__ void dft_small<6>(float2 *v, float s) { dft_pfa<2, 3>(v, s); }
template <>
__device__ __forceinline__ void dft_small<10>(float2 *v, float s) { dft_pfa<2, 5>(v, s); }
template <>
__device__ __forceinline__ void dft_small<12>(float2 *v, float s) { dft_pfa<4, 3>(v, s); }
template <>
__device__ __forceinline__ void dft_small<15>(float2 *v, float s) { dft_pfa<3, 5>(v, s); }

// 9 = 3 x 3 (Cooley-Tukey): n = 3 n1 + n2, k = k1 + 3 k2; inner DFTs over n1, twiddle
// W9^(n2 k1), outer DFTs over n2.  cos/sin of 2 pi m / 9 for m = 1, 2, 4.
template <>
__device__ __forceinline__ void dft_small<9>(float2 *v, float s) {
    const float2 w1 = make_float2(0.76604444311897804f, s * 0.64278760968653933f);
    const float2 w2 = make_float2(0.17364817766693035f, s * 0.98480775301220806f);
    const float2 w4 = make_float2(-0.93969262078590838f, s * 0.34202014332566873f);
    float2 a[3][3];
#pragma unroll
    for (int n2 = 0; n2 < 3; n2++) {
        a[n2][0] = v[n2];
        a[n2][1] = v[3 + n2];
        a[n2][2] = v[6 + n2];
        dft_small<3>(a[n2], s);
    }
    a[1][1] = cmul(a[1][1], w1);
    a[1][2] = cmul(a[1][2], w2);
    a[2][1] = cmul(a[2][1], w2);
    a[2][2] = cmul(a[2][2], w4);
#pragma unroll
    for (int k1 = 0; k1 < 3; k1++) {
        float2 b[3] = {a[0][k1], a[1][k1], a[2][k1]};
        dft_small<3>(b, s);
        v[k1] = b[0];
        v[k1 + 3] = b[1];
        v[k1 + 6] = b[2];
    }
}

// One Stockham stage of radix P over `batch` transforms (buffers `stride` apart).
template <int P>
__device__ __forceinline__ void stage_fixed(const float2 *in, float2 *out, int n, int L, const float2 *tw,
                                            float s, int batch, int stride) {
    const int q = n / P;
    const int twstep = n / (L * P);
    const int total = batch * q;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int t = idx / q, j = idx - t * q;
        const float2 *src = in + t * stride;
        float2 *dst = out + t * stride;
        const int k = j % L;
        float2 v[P];
#pragma unroll
        for (int r = 0; r < P; r++) v[r] = src[j + r * q];
        if (k != 0) {
#pragma unroll
            for (int r = 1; r < P; r++) v[r] = cmul(v[r], tw_at(tw, r * k * twstep, s));
        }
        dft_small<P>(v, s);
        const int base = (j / L) * L * P + k;
#pragma unroll
        for (int r = 0; r < P; r++) dst[base + r * L] = v[r];
    }
}

// Direct p-point DFT (p odd) of butterfly j whose inputs src[j + r q] are already twiddled.  The
// symmetric pairs a_r = x_r + x_(p-r), b_r = x_r - x_(p-r) overwrite the inputs (each butterfly owns
// its inputs, and a stage's input buffer is dead after it); then X_qq and X_(p-qq) come together as
// x_0 + sum a_r cos(t) +- i s sum b_r sin(t), t = 2 pi (r qq mod p) / p, with cos and sin read from
// the length's table (entry (r qq mod p) q) and the exponent advanced by qq per term.
__device__ __forceinline__ void odd_dft_inplace(float2 *src, float2 *dst, int j, int q, int p, int L, int base,
                                                const float2 *tw, float s) {
    const int h = (p - 1) >> 1;
    const float2 x0 = src[j];
    float2 sum = x0;
    for (int r = 1; r <= h; r++) {
        const float2 u = src[j + r * q], v = src[j + (p - r) * q];
        const float2 a = cadd(u, v);
        src[j + r * q] = a;
        src[j + (p - r) * q] = csub(u, v);
        sum = cadd(sum, a);
    }
    dst[base] = sum;
    for (int qq = 1; qq <= h; qq++) {
        float2 re = x0, im = make_float2(0.f, 0.f);
        int e = 0;
        for (int r = 1; r <= h; r++) {
            e += qq;
            if (e >= p) e -= p;
            const float2 w = __ldg(tw + e * q);  // (cos t, -sin t)
            const float2 a = src[j + r * q], b = src[j + (p - r) * q];
            re.x = fmaf(a.x, w.x, re.x);
            re.y = fmaf(a.y, w.x, re.y);
            im.x = fmaf(b.x, -w.y, im.x);
            im.y = fmaf(b.y, -w.y, im.y);
        }
        dst[base + qq * L] = make_float2(re.x - s * im.y, re.y + s * im.x);
        dst[base + (p - qq) * L] = make_float2(re.x + s * im.y, re.y - s * im.x);
    }
}

// Radix-p stage for an odd prime p <= FFT_MAX_GENERIC without a register kernel.
__device__ __forceinline__ void stage_generic(float2 *in, float2 *out, int n, int L, int p,
                                              const float2 *tw, float s, int batch, int stride) {
    const int q = n / p;
    const int twstep = n / (L * p);
    const int total = batch * q;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int t = idx / q, j = idx - t * q;
        float2 *src = in + t * stride;
        float2 *dst = out + t * stride;
        const int k = j % L;
        const int base = (j / L) * L * p + k;
        if (k != 0)
            for (int r = 1; r < p; r++) src[j + r * q] = cmul(src[j + r * q], tw_at(tw, r * k * twstep, s));
        odd_dft_inplace(src, dst, j, q, p, L, base, tw, s);
    }
}

// Stockham FFT of `batch` transforms of length n (no Bluestein), ping-ponging between a and b.
// Returns the buffer holding the result.  Every thread of the block must call it.
__device__ inline float2 *fft_stockham(float2 *a, float2 *b, int n, int nst, const int *radix, const float2 *tw,
                                       float s, int batch, int stride) {
    int L = 1;
    float2 *in = a, *out = b;
    for (int st = 0; st < nst; st++) {
        const int p = radix[st];
        __syncthreads();
        switch (p) {
            case 2: stage_fixed<2>(in, out, n, L, tw, s, batch, stride); break;
            case 3: stage_fixed<3>(in, out, n, L, tw, s, batch, stride); break;
            case 4: stage_fixed<4>(in, out, n, L, tw, s, batch, stride); break;
            case 5: stage_fixed<5>(in, out, n, L, tw, s, batch, stride); break;
            case 6: stage_fixed<6>(in, out, n, L, tw, s, batch, stride); break;
            case 8: stage_fixed<8>(in, out, n, L, tw, s, batch, stride); break;
            case 9: stage_fixed<9>(in, out, n, L, tw, s, batch, stride); break;
            case 10: stage_fixed<10>(in, out, n, L, tw, s, batch, stride); break;
            case 12: stage_fixed<12>(in, out, n, L, tw, s, batch, stride); break;
            case 15: stage_fixed<15>(in, out, n, L, tw, s, batch, stride); break;
            default: stage_generic(in, out, n, L, p, tw, s, batch, stride); break;
        }
        L *= p;
        float2 *t = in;
        in = out;
        out = t;
    }
    __syncthreads();
    return in;
}

// Shared-memory floats a transform of this length needs per batch entry (two ping-pong buffers).
__host__ __device__ inline int fft_work_len(const FftLen &P) { return P.bluestein ? P.m : P.n; }

// FFT of `batch` transforms of length P.n stored in a (stride apart, stride >= fft_work_len);
// b is scratch of the same size.  Result (unscaled) returned in a or b.
__device__ inline float2 *fft_run(float2 *a, float2 *b, const FftLen &P, float s, int batch, int stride) {
    if (!P.bluestein) return fft_stockham(a, b, P.n, P.nst, P.radix, P.tw, s, batch, stride);
    const int n = P.n, m = P.m;
    // a_j = x_j * c_j (c conjugated for the inverse sign), zero padded to m
    __syncthreads();
    for (int idx = threadIdx.x; idx < batch * m; idx += blockDim.x) {
        const int t = idx / m, j = idx - t * m;
        float2 *x = a + t * stride;
        if (j < n) {
            float2 c = __ldg(P.chirp + j);
            if (s > 0) c = conjf2(c);
            x[j] = cmul(x[j], c);
        } else {
            x[j] = make_float2(0.f, 0.f);
        }
    }
    float2 *r = fft_stockham(a, b, m, P.mst, P.mradix, P.mtw, -1.f, batch, stride);
    const float2 *B = s < 0 ? P.bfwd : P.binv;
    for (int idx = threadIdx.x; idx < batch * m; idx += blockDim.x) {
        const int t = idx / m, j = idx - t * m;
        r[t * stride + j] = cmul(r[t * stride + j], __ldg(B + j));
    }
    float2 *o = (r == a) ? b : a;
    float2 *y = fft_stockham(r, o, m, P.mst, P.mradix, P.mtw, 1.f, batch, stride);
    for (int idx = threadIdx.x; idx < batch * n; idx += blockDim.x) {
        const int t = idx / n, j = idx - t * n;
        float2 c = __ldg(P.chirp + j);
        if (s > 0) c = conjf2(c);
        y[t * stride + j] = cmul(y[t * stride + j], c);
    }
    __syncthreads();
    return y;
}

// ---------------------------------------------------------------------------------------------
// Warp-level engine: a warp transforms nb sequences (stored wl apart) with __syncwarp between
// stages only, so the warps of a CTA progress independently.  Stage twiddles are read from `stw`
// (usually a shared-memory copy of FftLen::stw), laid out [k][r-1] so each butterfly reads a
// contiguous run.  Integer quotients use floor((i + 0.5) * (1/d)) in float, exact for i < 2^22.

template <int P>
__device__ __forceinline__ void warp_stage(const float2 *in, float2 *out, int n, int L, float invL, float invq,
                                           const float2 *stw, float s, int nb, int wl) {
    const int q = n / P;
    for (int idx = threadIdx.x & 31; idx < nb * q; idx += 32) {
        const int t = nb > 1 ? __float2int_rz((float(idx) + 0.5f) * invq) : 0;
        const int j = idx - t * q;
        const float2 *src = in + t * wl;
        float2 *dst = out + t * wl;
        const int jl = __float2int_rz((float(j) + 0.5f) * invL);
        const int k = j - jl * L;
        float2 v[P];
#pragma unroll
        for (int r = 0; r < P; r++) v[r] = src[j + r * q];
        if (k != 0) {
            const float2 *w = stw + k * (P - 1) - 1;
#pragma unroll
            for (int r = 1; r < P; r++) v[r] = cmul(v[r], make_float2(w[r].x, -s * w[r].y));
        }
        dft_small<P>(v, s);
        const int base = jl * L * P + k;
#pragma unroll
        for (int r = 0; r < P; r++) dst[base + r * L] = v[r];
    }
}

// odd prime radix without a register kernel: twiddle in place, then the direct p-point DFT
__device__ __forceinline__ void warp_stage_generic(float2 *in, float2 *out, int n, int L, float invL,
                                                   float invq, int p, const float2 *stw, const float2 *tw, float s,
                                                   int nb, int wl) {
    const int q = n / p;
    for (int idx = threadIdx.x & 31; idx < nb * q; idx += 32) {
        const int t = nb > 1 ? __float2int_rz((float(idx) + 0.5f) * invq) : 0;
        const int j = idx - t * q;
        float2 *src = in + t * wl;
        float2 *dst = out + t * wl;
        const int jl = __float2int_rz((float(j) + 0.5f) * invL);
        const int k = j - jl * L;
        const int base = jl * L * p + k;
        if (k != 0) {
            for (int r = 1; r < p; r++) {
                const float2 w = stw[k * (p - 1) + r - 1];
                src[j + r * q] = cmul(src[j + r * q], make_float2(w.x, -s * w.y));
            }
        }
        odd_dft_inplace(src, dst, j, q, p, L, base, tw, s);
    }
}

__device__ inline float2 *warp_stockham(float2 *a, float2 *b, int n, int nst, const int *radix, const int *stride,
                                        const float *inv_stride, const float *inv_q, const int *stw_off,
                                        const float2 *stw, const float2 *tw, float s, int nb, int wl) {
    float2 *in = a, *out = b;
    for (int st = 0; st < nst; st++) {
        const int p = radix[st], L = stride[st];
        const float invL = inv_stride[st], iq = inv_q[st];
        const float2 *w = stw + stw_off[st];
        __syncwarp();
        switch (p) {
            case 2: warp_stage<2>(in, out, n, L, invL, iq, w, s, nb, wl); break;
            case 3: warp_stage<3>(in, out, n, L, invL, iq, w, s, nb, wl); break;
            case 4: warp_stage<4>(in, out, n, L, invL, iq, w, s, nb, wl); break;
            case 5: warp_stage<5>(in, out, n, L, invL, iq, w, s, nb, wl); break;
            case 6: warp_stage<6>(in, out, n, L, invL, iq, w, s, nb, wl); break;
            case 8: warp_stage<8>(in, out, n, L, invL, iq, w, s, nb, wl); break;
            case 9: warp_stage<9>(in, out, n, L, invL, iq, w, s, nb, wl); break;
            case 10: warp_stage<10>(in, out, n, L, invL, iq, w, s, nb, wl); break;
            case 12: warp_stage<12>(in, out, n, L, invL, iq, w, s, nb, wl); break;
            case 15: warp_stage<15>(in, out, n, L, invL, iq, w, s, nb, wl); break;
            default: warp_stage_generic(in, out, n, L, invL, iq, p, w, tw, s, nb, wl); break;
        }
        float2 *t = in;
        in = out;
        out = t;
    }
    __syncwarp();
    return in;
}

// Copies the stage twiddles of P into shared memory (all threads of the block; call before a
// __syncthreads).  Returns the entries copied.
__device__ inline void stage_twiddles_to_shared(const FftLen &P, float2 *dst) {
    const float2 *src = P.bluestein ? P.mstw : P.stw;
    const int len = P.bluestein ? P.mstw_len : P.stw_len;
    for (int i = threadIdx.x; i < len; i += blockDim.x) dst[i] = __ldg(src + i);
}
__host__ __device__ inline int stage_twiddle_len(const FftLen &P) { return P.bluestein ? P.mstw_len : P.stw_len; }

// nb transforms of length P.n held at a + t*wl (t < nb) by the calling warp (b: scratch of the same
// shape; wl >= fft_work_len(P)).  `stw` is the stage-twiddle table (shared copy or P.stw / P.mstw).
// Returns the buffer with the unscaled results.
__device__ inline float2 *fft_warp(float2 *a, float2 *b, const FftLen &P, const float2 *stw, float s, int nb, int wl) {
    if (!P.bluestein)
        return warp_stockham(a, b, P.n, P.nst, P.radix, P.stride, P.inv_stride, P.inv_q, P.stw_off, stw, P.tw, s, nb,
                             wl);
    const int n = P.n, m = P.m, lane = threadIdx.x & 31;
    __syncwarp();
    for (int t = 0; t < nb; t++)
        for (int j = lane; j < m; j += 32) {
            float2 *x = a + t * wl;
            if (j < n) {
                float2 c = __ldg(P.chirp + j);
                if (s > 0) c = conjf2(c);
                x[j] = cmul(x[j], c);
            } else {
                x[j] = make_float2(0.f, 0.f);
            }
        }
    float2 *r = warp_stockham(a, b, m, P.mst, P.mradix, P.mstride, P.minv_stride, P.minv_q, P.mstw_off, stw, P.mtw,
                              -1.f, nb, wl);
    const float2 *B = s < 0 ? P.bfwd : P.binv;
    for (int t = 0; t < nb; t++)
        for (int j = lane; j < m; j += 32) r[t * wl + j] = cmul(r[t * wl + j], __ldg(B + j));
    float2 *o = (r == a) ? b : a;
    float2 *y = warp_stockham(r, o, m, P.mst, P.mradix, P.mstride, P.minv_stride, P.minv_q, P.mstw_off, stw, P.mtw,
                              1.f, nb, wl);
    for (int t = 0; t < nb; t++)
        for (int j = lane; j < n; j += 32) {
            float2 c = __ldg(P.chirp + j);
            if (s > 0) c = conjf2(c);
            y[t * wl + j] = cmul(y[t * wl + j], c);
        }
    __syncwarp();
    return y;
}

}  // namespace iqm

namespace iqm {

// ---------------------------------------------------------------------------------------------
// Fixed-length warp engine: the radix sequence is a template parameter pack, so every stride,
// quotient and loop bound is a compile-time constant and the butterflies carry no runtime index
// arithmetic beyond the lane number.  Same stage rule and twiddle layout as the runtime engine.
template <int N, int L, int... Rs>
struct FixedStages;

template <int N, int L>
struct FixedStages<N, L> {
    static __device__ __forceinline__ float2 *run(float2 *in, float2 *out, const float2 *, int, float) {
        __syncwarp();
        return in;
    }
};

template <int N, int L, int P, int... Rs>
struct FixedStages<N, L, P, Rs...> {
    static __device__ __forceinline__ float2 *run(float2 *in, float2 *out, const float2 *stw, int stw_off, float s) {
        constexpr int Q = N / P;
        __syncwarp();
        const int lane = threadIdx.x & 31;
#pragma unroll
        for (int it = 0; it < (Q + 31) / 32; it++) {
            const int j = lane + 32 * it;
            if ((Q % 32 == 0) || j < Q) {
                const int jl = j / L, k = j - jl * L;
                float2 v[P];
#pragma unroll
                for (int r = 0; r < P; r++) v[r] = in[j + r * Q];
                if (L > 1 && k != 0) {
                    const float2 *w = stw + stw_off + k * (P - 1) - 1;
#pragma unroll
                    for (int r = 1; r < P; r++) v[r] = cmul(v[r], make_float2(w[r].x, -s * w[r].y));
                }
                dft_small<P>(v, s);
                const int base = jl * L * P + k;
#pragma unroll
                for (int r = 0; r < P; r++) out[base + r * L] = v[r];
            }
        }
        return FixedStages<N, L * P, Rs...>::run(out, in, stw, stw_off + (P - 1) * L, s);
    }
};

// Plan types: a length and its radix sequence (must match what the host planner picks for N,
// since the stage-twiddle table is laid out for that sequence).
template <int N, int... Rs>
struct FixedPlan {
    static constexpr int n = N;
    static __device__ __forceinline__ float2 *run(float2 *a, float2 *b, const float2 *stw, float s) {
        return FixedStages<N, 1, Rs...>::run(a, b, stw, 0, s);
    }
};


// In-place form of the fixed-length engine: every stage first reads all of a lane's butterfly inputs
// into registers, synchronises the warp, then writes the butterflies' outputs into the same buffer
// (the same values the two-buffer stage would write), so one transform needs one buffer of N points.
template <int N, int L, int... Rs>
struct FixedStagesIP;

template <int N, int L>
struct FixedStagesIP<N, L> {
    static __device__ __forceinline__ void run(float2 *, const float2 *, int, float) {}
};

template <int N, int L, int P, int... Rs>
struct FixedStagesIP<N, L, P, Rs...> {
    static __device__ __forceinline__ void run(float2 *buf, const float2 *stw, int stw_off, float s) {
        constexpr int Q = N / P;
        constexpr int IT = (Q + 31) / 32;
        const int lane = threadIdx.x & 31;
        float2 v[IT][P];
#pragma unroll
        for (int it = 0; it < IT; it++) {
            const int j = lane + 32 * it;
            if ((Q % 32 == 0) || j < Q) {
#pragma unroll
                for (int r = 0; r < P; r++) v[it][r] = buf[j + r * Q];
            }
        }
        __syncwarp();
#pragma unroll
        for (int it = 0; it < IT; it++) {
            const int j = lane + 32 * it;
            if ((Q % 32 == 0) || j < Q) {
                const int jl = j / L, k = j - jl * L;
                if (L > 1 && k != 0) {
                    const float2 *w = stw + stw_off + k * (P - 1) - 1;
#pragma unroll
                    for (int r = 1; r < P; r++) v[it][r] = cmul(v[it][r], make_float2(w[r].x, -s * w[r].y));
                }
                dft_small<P>(v[it], s);
                const int base = jl * L * P + k;
#pragma unroll
                for (int r = 0; r < P; r++) buf[base + r * L] = v[it][r];
            }
        }
        __syncwarp();
        FixedStagesIP<N, L * P, Rs...>::run(buf, stw, stw_off + (P - 1) * L, s);
    }
};

template <int N, int... Rs>
struct FixedPlanIP {
    static constexpr int n = N;
    // result in `a`; `b` is not used
    static __device__ __forceinline__ float2 *run(float2 *a, float2 *, const float2 *stw, float s) {
        __syncwarp();
        FixedStagesIP<N, 1, Rs...>::run(a, stw, 0, s);
        return a;
    }
};

}  // namespace iqm
