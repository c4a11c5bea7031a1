// Accuracy check of the SFU-based helpers in iqm_internal.cuh (cube root, power, square root,
// reciprocal) that the kernels use in place of CUDA's cbrtf, powf, sqrtf and IEEE division.  Both the
// helpers and CUDA's own functions run on the GPU over the same seeded inputs; the host compares each
// against a double-precision reference and prints, per function,
//   "<name> <largest relative error of the helper> <largest relative error of CUDA's function> <exact>"
// where <exact> is 1 when every special case (zero arguments) gave its required value.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "iqm_internal.cuh"

namespace {

__global__ void eval(int kind, const float *x, const float *y, int n, float *ours, float *cuda) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float a = x[i], b = y[i];
    switch (kind) {
        case 0: ours[i] = iqm::cbrt_pos(a); cuda[i] = cbrtf(a); break;
        case 1: ours[i] = iqm::pow_nonneg(a, b); cuda[i] = powf(a, b); break;
        case 2: ours[i] = iqm::sqrt_nonneg(a); cuda[i] = sqrtf(a); break;
        default: ours[i] = iqm::rcp_approx(a); cuda[i] = 1.0f / a; break;
    }
}

struct Lcg {  // deterministic inputs
    uint64_t s;
    double next() {
        s = s * 6364136223846793005ULL + 1442695040888963407ULL;
        return double(s >> 11) * (1.0 / 9007199254740992.0);
    }
};

float log_uniform(Lcg &g, double lo, double hi) { return float(std::exp(std::log(lo) + g.next() * std::log(hi / lo))); }

int check(int kind, const char *name, const std::vector<float> &x, const std::vector<float> &y) {
    const int n = int(x.size());
    float *dx, *dy, *d1, *d2;
    if (cudaMalloc(&dx, n * 4) || cudaMalloc(&dy, n * 4) || cudaMalloc(&d1, n * 4) || cudaMalloc(&d2, n * 4)) return 1;
    cudaMemcpy(dx, x.data(), n * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(dy, y.data(), n * 4, cudaMemcpyHostToDevice);
    eval<<<(n + 255) / 256, 256>>>(kind, dx, dy, n, d1, d2);
    if (cudaDeviceSynchronize() != cudaSuccess) return 1;
    std::vector<float> ours(n), cuda(n);
    cudaMemcpy(ours.data(), d1, n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(cuda.data(), d2, n * 4, cudaMemcpyDeviceToHost);
    cudaFree(dx); cudaFree(dy); cudaFree(d1); cudaFree(d2);
    double e_ours = 0.0, e_cuda = 0.0;
    int exact = 1;
    for (int i = 0; i < n; i++) {
        const double a = x[i], b = y[i];
        const double ref = kind == 0 ? std::cbrt(a) : kind == 1 ? std::pow(a, b) : kind == 2 ? std::sqrt(a) : 1.0 / a;
        if (ref == 0.0 || a == 0.0) {  // special cases: pow(0, y) and sqrt(0) must be exact
            if (double(ours[i]) != ref) exact = 0;
            continue;
        }
        e_ours = std::fmax(e_ours, std::fabs(double(ours[i]) - ref) / std::fabs(ref));
        e_cuda = std::fmax(e_cuda, std::fabs(double(cuda[i]) - ref) / std::fabs(ref));
    }
    std::printf("%s %.3e %.3e %d\n", name, e_ours, e_cuda, exact);
    return 0;
}

}  // namespace

int main() {
    const int N = 1 << 20;
    Lcg g{12345};
    std::vector<float> x(N), y(N, 0.0f);
    // cube root: the L*a*b* companding's range (0.008856, 1.1], then six decades either side of 1
    for (int i = 0; i < N; i++) x[i] = i < N / 2 ? float(0.008856 + g.next() * (1.1 - 0.008856)) : log_uniform(g, 1e-6, 1e6);
    if (check(0, "cbrt", x, y)) return 1;
    // power: bases over twelve decades with exponents in [0, 1] (FLIP raises HyAB distances to 0.7
    // and its colour error in [0, 1] to 1 - feature error), plus pow(0, y) for y = 0, 0.5, 1
    for (int i = 0; i < N; i++) {
        x[i] = log_uniform(g, 1e-9, 1e3);
        y[i] = i % 4 == 0 ? 0.7f : float(g.next());
    }
    x[0] = 0.0f; y[0] = 0.0f;
    x[1] = 0.0f; y[1] = 0.5f;
    x[2] = 0.0f; y[2] = 1.0f;
    if (check(1, "pow", x, y)) return 1;
    // square root: sums of squared filter responses and colour differences over forty decades, and 0
    for (int i = 0; i < N; i++) x[i] = log_uniform(g, 1e-20, 1e20);
    x[0] = 0.0f;
    if (check(2, "sqrt", x, y)) return 1;
    // reciprocal: the denominators the kernels invert (all normal, positive)
    for (int i = 0; i < N; i++) x[i] = log_uniform(g, 1e-20, 1e20);
    if (check(3, "rcp", x, y)) return 1;
    return 0;
}
