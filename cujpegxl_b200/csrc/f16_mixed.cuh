// Mixed-precision FP16-input arithmetic with FP32 results (sm_100), used by
// the fused frontend's chroma-from-luma sums; checked against
// convert-then-FP32 arithmetic by tests/gpu_checks/f16_mixed_check.cu.
#pragma once

#include <cuda_fp16.h>

namespace jxb {

// Mixed-precision forms (sm_100): the FP16 operands are widened exactly inside
// the instruction, so fma_f16(a, b, c) is fmaf(float(a), float(b), c) and
// add_f16(a, c) is float(a) + c, each rounded once, without separate
// conversions.
__device__ __forceinline__ float fma_f16(unsigned short a, unsigned short b, float c) {
    float d;
    asm("fma.rn.f32.f16 %0, %1, %2, %3;" : "=f"(d) : "h"(a), "h"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float add_f16(unsigned short a, float c) {
    float d;
    asm("add.rn.f32.f16 %0, %1, %2;" : "=f"(d) : "h"(a), "f"(c));
    return d;
}

}  // namespace jxb
