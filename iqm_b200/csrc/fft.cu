// Host side of the shared-memory FFT engine (fft.cuh): per-length plans with device tables,
// cached on the context.
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

// Radix sequence for n (8s, then 4 or 2, then odd primes ascending); false when n has a prime
// factor above FFT_MAX_GENERIC.
bool factor(int n, std::vector<int> &r) {
    r.clear();
    int m = n;
    int twos = 0;
    while (m % 2 == 0) {
        m /= 2;
        twos++;
    }
    while (twos >= 3) {
        r.push_back(8);
        twos -= 3;
    }
    if (twos == 2) r.push_back(4);
    if (twos == 1) r.push_back(2);
    for (int p = 3; p <= m; p += 2) {
        while (m % p == 0) {
            if (p > FFT_MAX_GENERIC) return false;
            r.push_back(p);
            m /= p;
        }
    }
    return true;
}

// In-place radix-2 FFT in double (host), used only to precompute Bluestein kernels.
void host_fft_pow2(std::vector<std::complex<double>> &a, int sign) {
    const int n = int(a.size());
    for (int i = 1, j = 0; i < n; i++) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (int len = 2; len <= n; len <<= 1) {
        const double ang = sign * 2.0 * M_PI / len;
        const std::complex<double> wl(std::cos(ang), std::sin(ang));
        for (int i = 0; i < n; i += len) {
            std::complex<double> w(1.0, 0.0);
            for (int k = 0; k < len / 2; k++) {
                const std::complex<double> u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
                w *= wl;
            }
        }
    }
}

void table(std::vector<float2> &out, int n) {
    out.resize(n);
    for (int t = 0; t < n; t++) {
        const double a = 2.0 * M_PI * double(t) / double(n);
        out[t] = make_float2(float(std::cos(a)), float(-std::sin(a)));
    }
}

}  // namespace

const FftLen &fft_len(iqm_ctx *ctx, int n) {
    auto it = ctx->fft_plans.find(n);
    if (it != ctx->fft_plans.end()) return it->second->len;
    IQM_REQUIRE(n >= 1 && n <= 16384, "FFT length out of range: " + std::to_string(n));
    auto *plan = new FftPlan();
    FftLen &L = plan->len;
    L.n = n;
    std::vector<int> r;
    std::vector<float2> tw, mtw, chirp, bf, bi;
    table(tw, n);
    if (factor(n, r)) {
        L.bluestein = 0;
        L.nst = int(r.size());
        int st = 1;
        for (int i = 0; i < L.nst; i++) {
            L.radix[i] = r[i];
            L.stride[i] = st;
            L.inv_stride[i] = 1.0f / float(st);
            st *= r[i];
        }
    } else {
        L.bluestein = 1;
        L.nst = 0;
        int m = 1;
        while (m < 2 * n - 1) m <<= 1;
        L.m = m;
        factor(m, r);
        L.mst = int(r.size());
        int st = 1;
        for (int i = 0; i < L.mst; i++) {
            L.mradix[i] = r[i];
            L.mstride[i] = st;
            L.minv_stride[i] = 1.0f / float(st);
            st *= r[i];
        }
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
            host_fft_pow2(b, -1);
            auto &dst = pass == 0 ? bf : bi;
            dst.resize(m);
            for (int k = 0; k < m; k++) dst[k] = make_float2(float(b[k].real() / m), float(b[k].imag() / m));
        }
    }
    const size_t bytes = sizeof(float2) * (tw.size() + mtw.size() + chirp.size() + bf.size() + bi.size());
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
    ctx->fft_plans[n] = plan;
    return L;
}

}  // namespace iqm

void iqm_release_fft_plans(iqm_ctx *ctx) {
    for (auto &kv : ctx->fft_plans) delete kv.second;
    ctx->fft_plans.clear();
}
