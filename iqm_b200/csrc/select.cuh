// Exact order statistics of non-negative FP32 values on the GPU (one CTA per array).
//
// Used where the reference sorts on the host and takes element [n/2]:
//   M-SVD median of block distances  (src/gpu/svd/svd.cpp:140-144)
//   FSIM noise median of |EO|^2      (src/gpu/fsim/steps/fsim_noise_power.cpp:193-203)
// For non-negative IEEE floats the bit pattern read as uint32 orders exactly like the value, so a
// three-digit radix select (12 + 10 + 10 bits) over those patterns returns the same element a full
// ascending sort would put at index k.
#pragma once

#include <cstdint>

namespace iqm {

constexpr int SELECT_BINS = 4096;

namespace detail {

constexpr int SELECT_UNROLL = 2;  // two quads in flight per thread fit 32 registers
// Padding past n: the bit pattern of a negative NaN, never among the non-negative inputs.
constexpr unsigned SELECT_PAD = 0xffffffffu;

// Loads the thread's SELECT_UNROLL quads of the block iteration starting at quad b0 (16-byte loads
// when v is 16-byte aligned and the quad is whole; SELECT_PAD past n).
__device__ __forceinline__ void load_quads(const float *__restrict__ v, int n, int nq, bool aligned, int b0,
                                           uint4 (&u)[SELECT_UNROLL]) {
#pragma unroll
    for (int r = 0; r < SELECT_UNROLL; r++) {
        const int q = b0 + r * blockDim.x + threadIdx.x;
        const int i = 4 * q;
        u[r] = make_uint4(SELECT_PAD, SELECT_PAD, SELECT_PAD, SELECT_PAD);
        if (q < nq) {
            if (aligned && i + 4 <= n) {
                u[r] = __ldcg(reinterpret_cast<const uint4 *>(v) + q);
            } else {
                if (i < n) u[r].x = __float_as_uint(__ldcg(v + i));
                if (i + 1 < n) u[r].y = __float_as_uint(__ldcg(v + i + 1));
                if (i + 2 < n) u[r].z = __float_as_uint(__ldcg(v + i + 2));
                if (i + 3 < n) u[r].w = __float_as_uint(__ldcg(v + i + 3));
            }
        }
    }
}

// Calls f(bits, valid) for every element of v[0..n), each thread's loads of an iteration issued
// before any call; `valid` is false for the padding.  The trip count is the same for all threads of
// the block, so f may use full-warp intrinsics.
template <typename F>
__device__ __forceinline__ void for_each_quad(const float *__restrict__ v, int n, F f) {
    const int nq = (n + 3) >> 2;
    const bool aligned = (reinterpret_cast<uintptr_t>(v) & 15u) == 0;
    for (int b0 = 0; b0 < nq; b0 += SELECT_UNROLL * blockDim.x) {
        uint4 u[SELECT_UNROLL];
        load_quads(v, n, nq, aligned, b0, u);
#pragma unroll
        for (int r = 0; r < SELECT_UNROLL; r++) {
            f(u[r].x, u[r].x != SELECT_PAD);
            f(u[r].y, u[r].y != SELECT_PAD);
            f(u[r].z, u[r].z != SELECT_PAD);
            f(u[r].w, u[r].w != SELECT_PAD);
        }
    }
}

// Block-wide: appends every element of v[0..n) whose bits >> sh equal `digit` to buf (in no
// particular order), counting in *count.  Each thread counts its matches among its quads, a warp scan
// turns the counts into slots, and one atomic per warp and iteration reserves them.  The caller
// guarantees that the matches fit buf.
__device__ __forceinline__ void gather_digit(const float *__restrict__ v, int n, int sh, unsigned digit,
                                             unsigned *buf, unsigned *count) {
    const int nq = (n + 3) >> 2;
    const bool aligned = (reinterpret_cast<uintptr_t>(v) & 15u) == 0;
    const int lane = threadIdx.x & 31;
    auto hit = [&](unsigned x) { return x != SELECT_PAD && (x >> sh) == digit; };
    for (int b0 = 0; b0 < nq; b0 += SELECT_UNROLL * blockDim.x) {
        uint4 u[SELECT_UNROLL];
        load_quads(v, n, nq, aligned, b0, u);
        unsigned cnt = 0;
#pragma unroll
        for (int r = 0; r < SELECT_UNROLL; r++)
            cnt += unsigned(hit(u[r].x)) + unsigned(hit(u[r].y)) + unsigned(hit(u[r].z)) + unsigned(hit(u[r].w));
        unsigned incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const unsigned total = __shfl_sync(0xffffffffu, incl, 31);
        if (total == 0u) continue;  // warp-uniform
        unsigned base = 0u;
        if (lane == 31) base = atomicAdd(count, total);
        unsigned pos = __shfl_sync(0xffffffffu, base, 31) + incl - cnt;
        if (cnt == 0u) continue;
#pragma unroll
        for (int r = 0; r < SELECT_UNROLL; r++) {
            if (hit(u[r].x)) buf[pos++] = u[r].x;
            if (hit(u[r].y)) buf[pos++] = u[r].y;
            if (hit(u[r].z)) buf[pos++] = u[r].z;
            if (hit(u[r].w)) buf[pos++] = u[r].w;
        }
    }
}

// Block-wide: finds the digit (bits >> sh) & dm of the k-th smallest element among those whose bits
// match `prefix` under `mask`, given their histogram of that digit in hist[]; updates the shared
// prefix, mask and k.
__device__ __forceinline__ void select_digit(const unsigned *hist, int bins, int sh, unsigned dm, unsigned prefix,
                                             unsigned mask, unsigned *s_prefix, unsigned *s_mask, unsigned *s_k,
                                             unsigned *s_warp_tot) {
    const int tid = threadIdx.x, nt = blockDim.x;
    // exclusive scan over bins: each thread owns a contiguous run of bins
    const int per = (bins + nt - 1) / nt;
    const int b0 = tid * per;
    unsigned local = 0;
    for (int b = b0; b < b0 + per && b < bins; b++) local += hist[b];
    unsigned incl = local;
    const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp_tot[wid] = incl;
    __syncthreads();
    unsigned before = 0;
    for (int w = 0; w < wid; w++) before += s_warp_tot[w];
    unsigned run = before + incl - local;  // count of values in bins < b0
    const unsigned kk = *s_k;
    __syncthreads();
    if (kk >= run && kk < run + local) {
        for (int b = b0; b < b0 + per && b < bins; b++) {
            const unsigned c = hist[b];
            if (kk < run + c) {
                *s_prefix = prefix | (unsigned(b) << sh);
                *s_mask = mask | (dm << sh);
                *s_k = kk - run;
                break;
            }
            run += c;
        }
    }
    __syncthreads();
}

}  // namespace detail

// Block-wide: returns the k-th smallest (0-based) of v[0..n) (all >= 0, no NaN).  `hist` is a
// shared array of SELECT_BINS counters.  With a shared buffer `buf` of `cap` words, the elements
// of the first digit's bucket are gathered there when they fit, and the last two digits are
// selected from shared memory (two reads of v instead of three).  Must be called by every thread
// of the block; blockDim.x must be a multiple of 32 and at most 1024.
__device__ inline float block_select_kth(const float *__restrict__ v, int n, int k, unsigned *hist,
                                         unsigned *buf = nullptr, int cap = 0) {
    __shared__ unsigned s_prefix, s_mask, s_k, s_count;
    __shared__ unsigned s_warp_tot[32];
    const int tid = threadIdx.x, nt = blockDim.x;
    if (tid == 0) {
        s_prefix = 0u;
        s_mask = 0u;
        s_k = unsigned(k);
        s_count = 0u;
    }
    constexpr int shifts[3] = {20, 10, 0};
    constexpr unsigned digit_masks[3] = {0xfffu, 0x3ffu, 0x3ffu};
    // first digit over v
    for (int b = tid; b < SELECT_BINS; b += nt) hist[b] = 0u;
    __syncthreads();
    detail::for_each_quad(v, n, [&](unsigned u, bool ok) {
        if (ok) atomicAdd(&hist[u >> shifts[0]], 1u);
    });
    __syncthreads();
    detail::select_digit(hist, SELECT_BINS, shifts[0], digit_masks[0], 0u, 0u, &s_prefix, &s_mask, &s_k, s_warp_tot);
    const unsigned bucket = s_prefix >> shifts[0];
    const bool staged = buf != nullptr && hist[bucket] <= unsigned(cap);  // uniform across the block
    __syncthreads();
    int m = n;
    if (staged) {
        // gather the bucket (hist[bucket] <= cap bounds every slot)
        detail::gather_digit(v, n, shifts[0], bucket, buf, &s_count);
        __syncthreads();
        m = int(s_count);
    }
#pragma unroll
    for (int pass = 1; pass < 3; pass++) {
        const int sh = shifts[pass];
        const unsigned dm = digit_masks[pass];
        for (int b = tid; b < SELECT_BINS; b += nt) hist[b] = 0u;
        __syncthreads();
        const unsigned prefix = s_prefix, mask = s_mask;
        if (staged) {
            for (int i = tid; i < m; i += nt) {
                const unsigned u = buf[i];
                if ((u & mask) == prefix) atomicAdd(&hist[(u >> sh) & dm], 1u);
            }
        } else {
            detail::for_each_quad(v, n, [&](unsigned u, bool ok) {
                if (ok && (u & mask) == prefix) atomicAdd(&hist[(u >> sh) & dm], 1u);
            });
        }
        __syncthreads();
        detail::select_digit(hist, int(dm) + 1, sh, dm, prefix, mask, &s_prefix, &s_mask, &s_k, s_warp_tot);
    }
    return __uint_as_float(s_prefix);
}

}  // namespace iqm
