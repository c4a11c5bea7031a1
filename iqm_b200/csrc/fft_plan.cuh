// Host access to cached per-length FFT plans (fft.cu).
#pragma once

#include "fft.cuh"
#include "iqm_internal.cuh"

namespace iqm {
// Plan of length n on this context (device tables created on first use, synchronously).
const FftLen &fft_len(iqm_ctx *ctx, int n);
}  // namespace iqm
