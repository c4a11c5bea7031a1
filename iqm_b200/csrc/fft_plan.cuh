// Host access to cached per-length FFT plans (fft.cu).
#pragma once

#include <vector>

#include "fft.cuh"
#include "iqm_internal.cuh"

namespace iqm {
// Host-side choice for length n: returns true with the radix sequence `r` for a direct transform,
// or false for Bluestein with its length `m` and m's radix sequence `rm` (r then holds n's direct
// sequence if one exists).  Pure host code, no device needed.
bool plan_length(int n, std::vector<int> &r, int &m, std::vector<int> &rm);

// Plan of length n on this context (device tables created on first use, synchronously).
const FftLen &fft_len(iqm_ctx *ctx, int n);
}  // namespace iqm
