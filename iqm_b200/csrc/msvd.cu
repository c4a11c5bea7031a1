// M-SVD on sm_100a.
//
// Reference path (cadik/IQM, src/gpu/svd/svd.cpp:39-164): on the host, OpenCV grey conversion
// (cv::cvtColor RGB2GRAY, uint8) and cv::SVD(NO_UV) of every 8x8 block of both images, for blocks
// with x+8 < W and y+8 < H only; on the GPU, the per-block distance D = sqrt(sum_k (s_k - r_k)^2)
// (shaders/svd/svd.glsl:24-54); on the host again a sort, the median D[n/2] and
// msvd = sum |D - median| / n with n = (W/8)*(H/8) (skipped slots count as D = 0).
//
// Here everything runs on the device in two kernels:
//   msvd_block_kernel  two lanes per block slot (one per image): 8 rows x 8 RGBA8 pixels straight
//                      into registers (two 16-byte loads per row, coalesced across a warp of
//                      horizontally adjacent blocks), OpenCV's 15-bit fixed-point grey, one-sided
//                      Jacobi SVD in registers (FP32 rotations, inner products and rotation test,
//                      two rows per packed FP32x2 instruction; FP64 final norms), D in FP32 as the
//                      shader does;
//   msvd_pool_kernel   one CTA per pair: exact median by radix select (select.cuh), then the mean
//                      absolute deviation summed in FP64, and the optional D/max(D) map.
#include <cfloat>
#include <cmath>

#include "iqm_internal.cuh"
#include "packed_f32x2.cuh"
#include "select.cuh"

namespace {

constexpr int BLOCK_THREADS = 128;
constexpr int POOL_THREADS = 1024;

struct MsvdPairDev {
    const uint8_t *a;
    const uint8_t *b;
    float *map;          // nullable, bw*bh
    long long pitch;
    int w, h;
    int bw, bh;          // W/8, H/8 block slots
    int vx, vy;          // computed blocks per row / column (x+8 < W, y+8 < H)
    int slot_base;       // first global slot of this pair
    int vec_ok;
};

struct MsvdArgs {
    const MsvdPairDev *pairs;
    int npairs;
    int total_slots;
    float *dist;         // total_slots
    double *scores;      // npairs
};

__device__ __forceinline__ float gray_u8(uint32_t px) {
    // cv::cvtColor(COLOR_RGB2GRAY) on 8-bit data: (R*9798 + G*19235 + B*3735 + 2^14) >> 15
    const uint32_t r = px & 0xffu, g = (px >> 8) & 0xffu, b = (px >> 16) & 0xffu;
    return float((r * 9798u + g * 19235u + b * 3735u + 16384u) >> 15);
}

__device__ __forceinline__ int find_pair(const MsvdPairDev *p, int n, int slot) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (p[mid].slot_base <= slot) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Loads one 8x8 grey block, column-major in registers as row pairs: c[col][k] = (row 2k, row 2k + 1).
__device__ __forceinline__ void load_block(const uint8_t *img, long long pitch, int x, int y, bool vec,
                                           float2 c[8][4]) {
#pragma unroll
    for (int r = 0; r < 8; r++) {
        const uint8_t *row = img + (long long)(y + r) * pitch + 4LL * x;
        uint32_t px[8];
        if (vec) {
            const uint4 lo = __ldg(reinterpret_cast<const uint4 *>(row));
            const uint4 hi = __ldg(reinterpret_cast<const uint4 *>(row) + 1);
            px[0] = lo.x; px[1] = lo.y; px[2] = lo.z; px[3] = lo.w;
            px[4] = hi.x; px[5] = hi.y; px[6] = hi.z; px[7] = hi.w;
        } else {
#pragma unroll
            for (int q = 0; q < 8; q++) px[q] = __ldg(reinterpret_cast<const uint32_t *>(row) + q);
        }
#pragma unroll
        for (int q = 0; q < 8; q++) {
            if (r & 1) c[q][r >> 1].y = gray_u8(px[q]);
            else c[q][r >> 1].x = gray_u8(px[q]);
        }
    }
}

// <ci, cj> over the 8 rows: the even and odd rows as the two halves of packed FMAs, then their sum
__device__ __forceinline__ float dot8(const float2 (&ci)[4], const float2 (&cj)[4]) {
    float2 q = iqm::mul2(ci[0], cj[0]);
#pragma unroll
    for (int k = 1; k < 4; k++) q = iqm::fma2(ci[k], cj[k], q);
    return q.x + q.y;
}

// Singular values (descending) of the 8x8 matrix whose columns are c[0..7]; c is destroyed.
// One-sided Jacobi: each (i, j) column pair is rotated so the columns become orthogonal.  Inner
// products, rotations and the squared column norms (recomputed from the rotated columns) are FP32,
// two rows per packed FP32x2 instruction (half the instructions and half the unrolled code of the
// sweep, which otherwise overflows the instruction cache); the rotation test
// |<ci,cj>|^2 > eps^2 |ci|^2 |cj|^2 is FP32 too (eps = 4 FLT_EPSILON, above FP32 rounding noise, so
// sweeps stop: at most 6 on the OpenCV fixture blocks), and the final norms are accumulated in FP64
// like OpenCV's Jacobi SVD.
__device__ __forceinline__ void svd8_values(float2 c[8][4], float s[8]) {
    float nrm[8];
#pragma unroll
    for (int i = 0; i < 8; i++) nrm[i] = dot8(c[i], c[i]);
    const float eps2 = 16.0f * FLT_EPSILON * FLT_EPSILON;
    for (int sweep = 0; sweep < 60; sweep++) {
        bool changed = false;
#pragma unroll
        for (int i = 0; i < 7; i++) {
#pragma unroll
            for (int j = i + 1; j < 8; j++) {
                const float p = dot8(c[i], c[j]);
                // all three products stay far inside FP32's range (norms < 2^20); pairs whose inner
                // product is below 1e-15 count as orthogonal, so columns that shrink to rounding
                // noise do not keep the sweeps going through denormal products
                if (p * p > fmaxf(eps2 * nrm[i] * nrm[j], 1e-30f)) {
                    // 1e-15 < |p| <= |ci||cj| < 2^20 here, so the SFU reciprocal is accurate to a few
                    // ulp; the angle only steers the sweep, later rotations remove what it leaves
                    const float zeta = (nrm[j] - nrm[i]) * iqm::rcp_approx(2.0f * p);
                    const float az = fabsf(zeta);
                    // tan(theta): smaller root of t^2 + 2 zeta t - 1 = 0 (1/(2 zeta) once zeta^2
                    // overflows); sqrt(z) as z rsqrt(z) for z = zeta^2 + 1 >= 1, and the SFU
                    // reciprocal of a denominator in [1, 2^61)
                    const float z = fmaf(zeta, zeta, 1.0f);
                    const float t = copysignf(1.0f, zeta) * iqm::rcp_approx(az < 1e18f ? az + z * iqm::rsqrt_approx(z) : 2.0f * az);
                    const float cs = iqm::rsqrt_approx(fmaf(t, t, 1.0f));
                    const float sn = cs * t;
                    const float2 cs2 = iqm::dup2(cs), sn2 = iqm::dup2(sn), msn2 = iqm::dup2(-sn);
                    float2 ni = iqm::dup2(0.f), nj = iqm::dup2(0.f);
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const float2 xi = c[i][k], xj = c[j][k];
                        const float2 yi = iqm::fma2(cs2, xi, iqm::mul2(msn2, xj));
                        const float2 yj = iqm::fma2(sn2, xi, iqm::mul2(cs2, xj));
                        c[i][k] = yi;
                        c[j][k] = yj;
                        ni = iqm::fma2(yi, yi, ni);
                        nj = iqm::fma2(yj, yj, nj);
                    }
                    nrm[i] = ni.x + ni.y;
                    nrm[j] = nj.x + nj.y;
                    changed = true;
                }
            }
        }
        if (!changed) break;
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
        double q = 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            q = fma(double(c[i][k].x), double(c[i][k].x), q);
            q = fma(double(c[i][k].y), double(c[i][k].y), q);
        }
        s[i] = float(sqrt(q));
    }
    // descending order (sorting network on 8 registers)
#define IQM_CSWAP(a, b)                         \
    do {                                        \
        const float hi_ = fmaxf(s[a], s[b]);    \
        const float lo_ = fminf(s[a], s[b]);    \
        s[a] = hi_;                             \
        s[b] = lo_;                             \
    } while (0)
    IQM_CSWAP(0, 1); IQM_CSWAP(2, 3); IQM_CSWAP(4, 5); IQM_CSWAP(6, 7);
    IQM_CSWAP(0, 2); IQM_CSWAP(1, 3); IQM_CSWAP(4, 6); IQM_CSWAP(5, 7);
    IQM_CSWAP(1, 2); IQM_CSWAP(5, 6); IQM_CSWAP(0, 4); IQM_CSWAP(3, 7);
    IQM_CSWAP(1, 5); IQM_CSWAP(2, 6);
    IQM_CSWAP(1, 4); IQM_CSWAP(3, 6);
    IQM_CSWAP(2, 4); IQM_CSWAP(3, 5);
    IQM_CSWAP(3, 4);
#undef IQM_CSWAP
}

// Two lanes per block slot: the even lane takes the block of the distorted image, the odd lane the
// same block of the reference; the odd lane's singular values reach the even lane by shuffle.  One
// copy of the SVD code serves both images and twice as many blocks are in flight.
// Five CTAs per SM (90 registers, no spills): with the packed row pairs, six CTAs at 80 registers
// spill the columns and measured 16% slower.
__global__ void __launch_bounds__(BLOCK_THREADS, 5) msvd_block_kernel(MsvdArgs args) {
    const int slot = (blockIdx.x * BLOCK_THREADS + threadIdx.x) >> 1;
    const int img = threadIdx.x & 1;
    const bool in_range = slot < args.total_slots;  // both lanes of a slot agree
    bool computed = false;
    MsvdPairDev P{};
    int bx = 0, by = 0;
    if (in_range) {
        P = args.pairs[find_pair(args.pairs, args.npairs, slot)];
        const int local = slot - P.slot_base;
        bx = local % P.bw;
        by = local / P.bw;
        computed = bx < P.vx && by < P.vy;  // other slots stay 0 (src/gpu/svd/svd.cpp:44,68-74)
    }
    // lanes that compute, fixed before the data-dependent sweeps (pairs of lanes agree)
    const unsigned mask = __ballot_sync(0xffffffffu, computed);
    if (computed) {
        {  // one 8x8 block of one image
            float2 c[8][4];
            load_block(img ? P.b : P.a, P.pitch, 8 * bx, 8 * by, P.vec_ok, c);
            float s[8];
            svd8_values(c, s);
            float acc = 0.0f;  // shaders/svd/svd.glsl:41-52: float, k = 0..7 in order
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const float sr = __shfl_xor_sync(mask, s[k], 1);
                const float t = s[k] - sr;
                acc = fmaf(t, t, acc);
            }
            if (!img) args.dist[slot] = sqrtf(acc);
        }
    }
    if (in_range && !computed && !img) args.dist[slot] = 0.0f;
}

__global__ void __launch_bounds__(POOL_THREADS) msvd_pool_kernel(MsvdArgs args) {
    __shared__ unsigned hist[iqm::SELECT_BINS];
    __shared__ double red_s[POOL_THREADS / 32];
    __shared__ float red_m[POOL_THREADS / 32];
    const MsvdPairDev &P = args.pairs[blockIdx.x];
    const int n = P.bw * P.bh;
    const float *D = args.dist + P.slot_base;
    const float med = iqm::block_select_kth(D, n, n / 2, hist);
    double s = 0.0;
    float mx = 0.0f;
    for (int i = threadIdx.x; i < n; i += POOL_THREADS) {
        const float v = __ldcg(D + i);
        s += double(fabsf(v - med));
        mx = fmaxf(mx, v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        mx = fmaxf(mx, __shfl_down_sync(0xffffffffu, mx, o));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        red_s[wid] = s;
        red_m[wid] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        float m = 0.0f;
        for (int w = 0; w < POOL_THREADS / 32; w++) {
            t += red_s[w];
            m = fmaxf(m, red_m[w]);
        }
        args.scores[blockIdx.x] = t / double(n);
        red_m[0] = m;
    }
    __syncthreads();
    if (P.map) {
        const float m = red_m[0];
        for (int i = threadIdx.x; i < n; i += POOL_THREADS) P.map[i] = __ldcg(D + i) / m;
    }
}

void msvd_enqueue(iqm_ctx *ctx, const std::vector<iqm_pair> &pairs, const std::vector<float *> &maps,
                  double *d_scores) {
    const int n = int(pairs.size());
    std::vector<MsvdPairDev> hd(n);
    long total = 0;
    for (int i = 0; i < n; i++) {
        const iqm_pair &q = pairs[i];
        MsvdPairDev &d = hd[i];
        d.a = q.input;
        d.b = q.ref;
        d.map = maps.empty() ? nullptr : maps[i];
        d.pitch = (long long)q.row_bytes;
        d.w = q.w;
        d.h = q.h;
        d.bw = q.w / 8;
        d.bh = q.h / 8;
        d.vx = q.w >= 9 ? (q.w - 1) / 8 : 0;  // x = 8*bx with x + 8 < W
        d.vy = q.h >= 9 ? (q.h - 1) / 8 : 0;
        d.slot_base = int(total);
        d.vec_ok = ((reinterpret_cast<uintptr_t>(q.input) | reinterpret_cast<uintptr_t>(q.ref) |
                     uintptr_t(q.row_bytes)) & 15u) == 0;
        total += long(d.bw) * d.bh;
    }
    IQM_REQUIRE(total < (1L << 31), "too many blocks in one batch");
    auto *d_desc = static_cast<MsvdPairDev *>(iqm::upload_bytes(ctx, ctx->desc, hd.data(), sizeof(MsvdPairDev) * n));
    MsvdArgs a{};
    a.pairs = d_desc;
    a.npairs = n;
    a.total_slots = int(total);
    a.dist = static_cast<float *>(ctx->scratch.get(sizeof(float) * size_t(total), ctx->stream));
    a.scores = d_scores;
    msvd_block_kernel<<<iqm::ceil_div(2 * total, BLOCK_THREADS), BLOCK_THREADS, 0, ctx->stream>>>(a);
    iqm::check_launch(ctx, "msvd_block_kernel");
    msvd_pool_kernel<<<n, POOL_THREADS, 0, ctx->stream>>>(a);
    iqm::check_launch(ctx, "msvd_pool_kernel");
}

}  // namespace

// The reference needs at least one 8x8 block slot: n = (W/8)*(H/8) > 0 (it divides by n).
static void check_msvd_pairs(const iqm_pair *pairs, int n) { iqm::check_pairs(pairs, n, 8, 8); }

void iqm::enqueue_msvd_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n, double *d_scores) {
    check_msvd_pairs(pairs, n);
    iqm::check_dev_alignment(pairs, n);
    IQM_REQUIRE(d_scores != nullptr, "d_scores is NULL");
    msvd_enqueue(ctx, std::vector<iqm_pair>(pairs, pairs + n), {}, d_scores);
}

extern "C" __attribute__((visibility("default"))) int iqm_msvd_dev(iqm_ctx *ctx, const iqm_pair *pairs, int n,
                                                                  double *d_scores) {
    return iqm::guarded(ctx, [&] { iqm::enqueue_msvd_dev(ctx, pairs, n, d_scores); });
}

extern "C" __attribute__((visibility("default"))) int iqm_msvd_batch(iqm_ctx *ctx, const iqm_pair *pairs, int n,
                                                                    double *scores) {
    return iqm::guarded(ctx, [&] {
        check_msvd_pairs(pairs, n);
        IQM_REQUIRE(scores != nullptr, "scores is NULL");
        auto *d_scores = static_cast<double *>(ctx->scores.get(sizeof(double) * n, ctx->stream));
        iqm::upload_pipelined(ctx, pairs, n, [&](const iqm_pair *dev, int first, int count) {
            msvd_enqueue(ctx, std::vector<iqm_pair>(dev, dev + count), {}, d_scores + first);
        });
        IQM_CHECK_CUDA(cudaMemcpyAsync(scores, d_scores, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
        IQM_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

extern "C" __attribute__((visibility("default"))) int iqm_msvd(iqm_ctx *ctx, const uint8_t *rgba_in,
                                                              const uint8_t *rgba_ref, int w, int h,
                                                              size_t row_bytes, float *block_map, double *msvd) {
    return iqm::guarded(ctx, [&] {
        IQM_REQUIRE(msvd != nullptr, "msvd is NULL");
        iqm_pair hp{rgba_in, rgba_ref, w, h, row_bytes};
        check_msvd_pairs(&hp, 1);
        auto dev = iqm::upload_pairs(ctx, &hp, 1);
        auto *d_score = static_cast<double *>(ctx->scores.get(sizeof(double), ctx->stream));
        const size_t nb = size_t(w / 8) * size_t(h / 8);
        std::vector<float *> maps;
        float *d_map = nullptr;
        if (block_map) {
            d_map = static_cast<float *>(ctx->maps.get(sizeof(float) * nb, ctx->stream));
            maps.push_back(d_map);
        }
        msvd_enqueue(ctx, dev, maps, d_score);
        IQM_CHECK_CUDA(cudaMemcpyAsync(msvd, d_score, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        if (block_map)
            IQM_CHECK_CUDA(cudaMemcpyAsync(block_map, d_map, sizeof(float) * nb, cudaMemcpyDeviceToHost, ctx->stream));
        IQM_CHECK_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}
