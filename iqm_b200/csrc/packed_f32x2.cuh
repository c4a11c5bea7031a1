// Packed FP32x2 arithmetic (sm_100 FFMA2 / FMUL2 / FADD2): one instruction does two independent FP32
// operations, each half rounded exactly like the scalar operation.
#pragma once

#include <cuda_runtime.h>

namespace iqm {

__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }

}  // namespace iqm
