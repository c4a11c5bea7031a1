// Host side of the shared-memory FFT engine (fft.cuh): per-length plans with device tables,
// cached on the context.
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

#include "fft.cuh"
#include "fft_plan.cuh"
#include "iqm_internal.cuh"

namespace iqm {

struct FftPlan {
    FftLen len{};
    void *dev = nullptr;  // all device tables of this length, one allocation
    ~FftPlan() {
        if (dev) cudaFree(dev);
    }
};

namespace {

// Radices the engines compute in registers, with an estimate of the instructions one butterfly
// costs a lane: loads and stores of its p points, p-1 twiddle loads and products, the p-point DFT
// itself and the per-iteration index work.
struct RegRadix {
    int p, cost;
};
const RegRadix kRegRadix[] = {{2, 23}, {3, 38}, {4, 49}, {5, 74}, {6, 83}, {8, 113},
                              {9, 164}, {10, 163}, {12, 185}, {15, 272}};

int butterfly_cost(int p) {
    for (const RegRadix &r : kRegRadix)
        if (r.p == p) return r.cost;
    return -1;
}

bool is_prime(int p) {
    if (p < 2) return false;
    for (int d = 2; d * d <= p; d++)
        if (p % d == 0) return false;
    return true;
}

// Radix sequence for n of least estimated warp time: a radix-p stage has n/p butterflies, which a
// warp runs 32 at a time, so it costs ceil(n / 32p) times the butterfly's cost, plus a fixed
// per-stage cost for the shared-memory round trip.  Odd primes up to FFT_MAX_GENERIC without a
// register kernel run as direct O(p^2) butterflies.  Odd radices come first so the first stage's
// strided writes avoid shared-memory bank conflicts.  False when n has a prime factor above
// FFT_MAX_GENERIC.
bool factor(int n, std::vector<int> &r, long long *total_cost = nullptr) {
    r.clear();
    if (n == 1) return true;
    constexpr long long kInf = 1LL << 50;
    std::vector<long long> cost(n + 1, kInf);
    std::vector<int> pick(n + 1, 0);
    cost[1] = 0;
    for (int m = 2; m <= n; m++) {
        if (n % m) continue;
        for (int p = 2; p <= m && p <= FFT_MAX_GENERIC; p++) {
            if (m % p || cost[m / p] >= kInf) continue;
            long long w = butterfly_cost(p);
            if (w < 0) {
                if (!is_prime(p)) continue;
                // in-place twiddles, symmetric pairs, then (p-1)^2/4 steps of 3 loads + 4 FMAs
                w = 10 + 11 * p + (7 * p * p) / 4;
            }
            const long long c = cost[m / p] + (long long)((n / p + 31) / 32) * w + 20;
            if (c < cost[m] || (c == cost[m] && p > pick[m])) {
                cost[m] = c;
                pick[m] = p;
            }
        }
    }
    if (cost[n] >= kInf) return false;
    if (total_cost) *total_cost = cost[n];
    for (int m = n; m > 1; m /= pick[m]) r.push_back(pick[m]);
    std::stable_sort(r.begin(), r.end(), [](int x, int y) { return (x & 1) > (y & 1); });
    return true;
}

// Stage parameters and stage twiddles W_{L p}^{r k} (sign -1) laid out [k][r-1].
void stage_tables(int n, const std::vector<int> &r, int *radix, int *stride, float *inv_stride, float *inv_q,
                  int *off, int &len, std::vector<float2> &stw) {
    int L = 1;
    len = 0;
    for (size_t i = 0; i < r.size(); i++) {
        const int p = r[i];
        radix[i] = p;
        stride[i] = L;
        inv_stride[i] = 1.0f / float(L);
        inv_q[i] = 1.0f / float(n / p);
        off[i] = len;
        for (int k = 0; k < L; k++)
            for (int q = 1; q < p; q++) {
                const double a = 2.0 * M_PI * double(q) * double(k) / double(L * p);
                stw.push_back(make_float2(float(std::cos(a)), float(-std::sin(a))));
            }
        len += (p - 1) * L;
        L *= p;
    }
}

// Mixed-radix DFT in double (host, decimation in time over the smallest prime factor), used only
// to precompute Bluestein kernels: out[k] = sum_t in[t stride] exp(sign 2 pi i t k / m).
void host_dft(const std::complex<double> *in, std::complex<double> *out, int m, int stride, int sign) {
    if (m == 1) {
        out[0] = in[0];
        return;
    }
    int p = 2;
    while (m % p) p++;
    const int q = m / p;
    std::vector<std::complex<double>> sub(m);
    for (int r = 0; r < p; r++) host_dft(in + r * stride, sub.data() + r * q, q, stride * p, sign);
    for (int k = 0; k < m; k++) {
        std::complex<double> acc = 0.0;
        for (int r = 0; r < p; r++) {
            const double a = sign * 2.0 * M_PI * double((long long)r * k % m) / double(m);
            acc += sub[r * q + k % q] * std::complex<double>(std::cos(a), std::sin(a));
        }
        out[k] = acc;
    }
}

bool smooth235(int m) {
    for (int p : {2, 3, 5})
        while (m % p == 0) m /= p;
    return m == 1;
}

void table(std::vector<float2> &out, int n) {
    out.resize(n);
    for (int t = 0; t < n; t++) {
        const double a = 2.0 * M_PI * double(t) / double(n);
        out[t] = make_float2(float(std::cos(a)), float(-std::sin(a)));
    }
}

}  // namespace

bool plan_length(int n, std::vector<int> &r, int &m, std::vector<int> &rm) {
    // Direct plan, or Bluestein on the smallest 2,3,5-smooth m >= 2n-1 when that is estimated
    // cheaper (two length-m transforms plus three pointwise passes).
    long long direct_cost = 0, m_cost = 0;
    const bool direct = factor(n, r, &direct_cost);
    m = 2 * n - 1;
    while (!smooth235(m)) m++;
    factor(m, rm, &m_cost);
    const long long blue_cost = 2 * m_cost + 3 * 12 * (long long)((m + 31) / 32);
    return direct && (n <= 2 || direct_cost <= blue_cost);
}

const FftLen &fft_len(iqm_ctx *ctx, int n) {
    auto it = ctx->fft_plans.find(n);
    if (it != ctx->fft_plans.end()) return it->second->len;
    IQM_REQUIRE(n >= 1 && n <= 16384, "FFT length out of range: " + std::to_string(n));
    auto *plan = new FftPlan();
    FftLen &L = plan->len;
    L.n = n;
    std::vector<int> r;
    std::vector<float2> tw, mtw, chirp, bf, bi, stw, mstw;
    table(tw, n);
    int m = 0;
    std::vector<int> rm;
    if (plan_length(n, r, m, rm)) {
        L.bluestein = 0;
        L.nst = int(r.size());
        stage_tables(n, r, L.radix, L.stride, L.inv_stride, L.inv_q, L.stw_off, L.stw_len, stw);
    } else {
        L.bluestein = 1;
        L.nst = 0;
        L.m = m;
        r = rm;
        L.mst = int(r.size());
        stage_tables(m, r, L.mradix, L.mstride, L.minv_stride, L.minv_q, L.mstw_off, L.mstw_len, mstw);
        table(mtw, m);
        chirp.resize(n);
        std::vector<std::complex<double>> c(n);
        for (int t = 0; t < n; t++) {
            const long long t2 = (long long)t * t % (2LL * n);
            const double a = -M_PI * double(t2) / double(n);
            c[t] = std::complex<double>(std::cos(a), std::sin(a));
            chirp[t] = make_float2(float(c[t].real()), float(c[t].imag()));
        }
        for (int pass = 0; pass < 2; pass++) {
            // pass 0: kernel conj(c) (forward transform); pass 1: kernel c (inverse transform)
            std::vector<std::complex<double>> b(m, 0.0);
            for (int d = 0; d < n; d++) {
                const std::complex<double> v = pass == 0 ? std::conj(c[d]) : c[d];
                b[d] = v;
                if (d) b[m - d] = v;
            }
            std::vector<std::complex<double>> bt(m);
            host_dft(b.data(), bt.data(), m, 1, -1);
            b.swap(bt);
            auto &dst = pass == 0 ? bf : bi;
            dst.resize(m);
            for (int k = 0; k < m; k++) dst[k] = make_float2(float(b[k].real() / m), float(b[k].imag() / m));
        }
    }
    IQM_REQUIRE(int(r.size()) <= FFT_MAX_STAGES, "FFT length needs too many stages");
    const size_t bytes =
        sizeof(float2) * (tw.size() + mtw.size() + chirp.size() + bf.size() + bi.size() + stw.size() + mstw.size());
    if (cudaMalloc(&plan->dev, bytes) != cudaSuccess) {
        cudaGetLastError();
        delete plan;
        throw Error{IQM_ENOMEM, "FFT table allocation failed"};
    }
    auto *p = static_cast<float2 *>(plan->dev);
    auto put = [&](const std::vector<float2> &v) -> const float2 * {
        if (v.empty()) return nullptr;
        const float2 *d = p;
        cudaMemcpy(p, v.data(), sizeof(float2) * v.size(), cudaMemcpyHostToDevice);
        p += v.size();
        return d;
    };
    L.tw = put(tw);
    L.mtw = put(mtw);
    L.chirp = put(chirp);
    L.bfwd = put(bf);
    L.binv = put(bi);
    L.stw = put(stw);
    L.mstw = put(mstw);
    ctx->fft_plans[n] = plan;
    return L;
}

}  // namespace iqm

void iqm_release_fft_plans(iqm_ctx *ctx) {
    for (auto &kv : ctx->fft_plans) delete kv.second;
    ctx->fft_plans.clear();
}
