// gt_simd.cuh -- packed FP32x2 arithmetic (sm_100a `*.rn.f32x2`) and the
// division by a fixed divisor used by the fast locate kernel.
//
// Each lane of an f32x2 instruction is an IEEE binary32 operation with
// round-to-nearest-even, exactly as the scalar instruction, so packing two
// independent accumulation chains into one register pair changes no bits.
#pragma once
#include <cuda_runtime.h>
#include "gt_internal.cuh"

namespace gt {

__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}

__device__ __forceinline__ float2 add2(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

__device__ __forceinline__ float2 mul2(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

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
