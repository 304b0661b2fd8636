// Correctly rounded division for the adaptive-quantisation ratios, on packed
// f32x2 arithmetic. Shared by the fused frontend and the exhaustive check in
// tests/gpu_checks/ratio_div_check.cu. Compiled with -fmad=false like every
// file here.
#pragma once

#include "xyb.cuh"

namespace jxb {

// a / b on both components, correctly rounded (bit-identical to IEEE
// division) for the adaptive-quantisation ratios below, by Markstein's method
// (P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34(1), 1990): the hardware
// reciprocal approximation, one Newton step on it, the quotient, its exact
// residual by FMA and one correction. Both operands are positive normal floats
// there (num >= kRatioEps, den >= kRatioVOffset); for every float argument v in
// [0, 4] of the ratio (it stays below 1.2: XYB Y <= 0.85, |X| small) the
// result was checked equal to IEEE division in both orientations, num/den and
// den/num (tests/gpu_checks/ratio_div_check.cu).
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float2 div2_ratio(float2 a, float2 b) {
    const float2 y{rcp_approx(b.x), rcp_approx(b.y)};
    const float2 nb{f2neg(b)};
    const float2 y1{__ffma2_rn(__ffma2_rn(nb, y, f2dup(1.0f)), y, y)};
    const float2 q{__fmul2_rn(a, y1)};
    return __ffma2_rn(__ffma2_rn(nb, q, a), y1, q);
}

}  // namespace jxb
