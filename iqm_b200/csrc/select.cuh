// Exact order statistics of non-negative FP32 values on the GPU (one CTA per array).
//
// Used where the reference sorts on the host and takes element [n/2]:
//   M-SVD median of block distances  (src/gpu/svd/svd.cpp:140-144)
//   FSIM noise median of |EO|^2      (src/gpu/fsim/steps/fsim_noise_power.cpp:193-203)
// For non-negative IEEE floats the bit pattern read as uint32 orders exactly like the value, so a
// three-pass radix select (11 + 11 + 10 bits) over those patterns returns the same element a full
// ascending sort would put at index k.
#pragma once

#include <cstdint>

namespace iqm {

constexpr int SELECT_BINS = 2048;

// Block-wide: returns the k-th smallest (0-based) of v[0..n) (all >= 0, no NaN).  `hist` is a
// shared array of SELECT_BINS counters.  Must be called by every thread of the block; blockDim.x
// must be a multiple of 32 and at most 1024.
__device__ inline float block_select_kth(const float *__restrict__ v, int n, int k, unsigned *hist) {
    __shared__ unsigned s_prefix, s_mask, s_k;
    __shared__ unsigned s_warp_tot[32];
    const int tid = threadIdx.x, nt = blockDim.x;
    if (tid == 0) {
        s_prefix = 0u;
        s_mask = 0u;
        s_k = unsigned(k);
    }
    const int shifts[3] = {21, 10, 0};
    const unsigned digit_masks[3] = {0x7ffu, 0x7ffu, 0x3ffu};
    for (int pass = 0; pass < 3; pass++) {
        const int sh = shifts[pass];
        const unsigned dm = digit_masks[pass];
        for (int b = tid; b < SELECT_BINS; b += nt) hist[b] = 0u;
        __syncthreads();
        const unsigned prefix = s_prefix, mask = s_mask;
        for (int i = tid; i < n; i += nt) {
            const unsigned u = __float_as_uint(v[i]);
            if ((u & mask) == prefix) atomicAdd(&hist[(u >> sh) & dm], 1u);
        }
        __syncthreads();
        // exclusive scan over bins: each thread owns a contiguous run of bins
        const int per = (SELECT_BINS + nt - 1) / nt;
        const int b0 = tid * per;
        unsigned local = 0;
        for (int b = b0; b < b0 + per && b < SELECT_BINS; b++) local += hist[b];
        unsigned incl = local;
        const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) s_warp_tot[wid] = incl;
        __syncthreads();
        unsigned before = 0;
        for (int w = 0; w < wid; w++) before += s_warp_tot[w];
        unsigned run = before + incl - local;  // count of values in bins < b0
        const unsigned kk = s_k;
        __syncthreads();
        if (kk >= run && kk < run + local) {
            for (int b = b0; b < b0 + per && b < SELECT_BINS; b++) {
                const unsigned c = hist[b];
                if (kk < run + c) {
                    s_prefix = prefix | (unsigned(b) << sh);
                    s_mask = mask | (dm << sh);
                    s_k = kk - run;
                    break;
                }
                run += c;
            }
        }
        __syncthreads();
    }
    return __uint_as_float(s_prefix);
}

}  // namespace iqm
