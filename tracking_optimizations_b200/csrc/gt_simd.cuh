// gt_simd.cuh -- packed FP32x2 arithmetic (sm_100a FFMA2/FADD2/FMUL2) and the
// division by a fixed divisor used by the fast locate kernel.
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
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }

// a / b for a divisor b known in advance, by Markstein's correction step
// (P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34(1), 1990): with y = RN(1/b),
// q = RN(a*y), the remainder r = a - q*b is exact under a fused
// multiply-add, and RN(q + r*y) is the correctly rounded quotient.  The host
// confirms the identity with IEEE division for every positive binary32
// dividend before a divisor is used on this path (verify_division_kernel).
__device__ __forceinline__ float2 div2(float2 a, FixedDiv f) {
    const float2 y = make_float2(f.y, f.y);
    const float2 nb = make_float2(f.nb, f.nb);
    const float2 q = mul2(a, y);
    const float2 r = fma2(q, nb, a);
    return fma2(r, y, q);
}

__device__ __forceinline__ float div1(float a, FixedDiv f) {
    const float q = __fmul_rn(a, f.y);
    const float r = __fmaf_rn(q, f.nb, a);
    return __fmaf_rn(r, f.y, q);
}

}  // namespace gt
