// gt_simd.cuh -- packed FP32x2 arithmetic (sm_100a FFMA2/FADD2/FMUL2) of the
// fast locate kernel.
//
// Each lane of an f32x2 instruction is an IEEE binary32 operation with
// round-to-nearest-even, exactly as the scalar instruction, so packing two
// independent accumulation chains into one register pair changes no bits.
#pragma once
#include <cuda_runtime.h>
#include "gt_internal.cuh"

namespace gt {

__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b as a fused multiply-add by -1: the product is exact, so the result
// is the correctly rounded difference, with no separate negation
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }

}  // namespace gt
