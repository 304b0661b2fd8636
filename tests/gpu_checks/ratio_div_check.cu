// Exhaustive check of div2_ratio (the adaptive-quantisation ratios' division)
// against IEEE division: for every float v in [0, 4], the ratio's numerator
// and denominator are formed as the frontend forms them (ratio_gamma on
// max(v, 0)), and both orientations are divided by div2_ratio (on the pair
// (v, next float)) and by div.rn. Prints the mismatch counts; exits 1 on any.
#include <cstdint>
#include <cstdio>

#include "ratio_div.cuh"

using namespace jxb;

__device__ __forceinline__ void num_den(float v, float& num, float& den) {
    const float v2{v * v};
    num = jx_fma(kRatioNumMul, v2, kRatioEps);
    den = jx_fma(kRatioDenMul * v, v2, kRatioVOffset);
}

__global__ void check(std::uint32_t lo, std::uint32_t hi, unsigned int* bad) {
    const std::uint32_t stride{gridDim.x * blockDim.x};
    for (std::uint32_t u{lo + blockIdx.x * blockDim.x + threadIdx.x}; u < hi; u += stride) {
        const float va{__uint_as_float(u)};
        const float vb{__uint_as_float(u + 1 < hi ? u + 1 : u)};
        float na, da, nb, db;
        num_den(va, na, da);
        num_den(vb, nb, db);
        const float2 q1{div2_ratio(make_float2(na, nb), make_float2(da, db))};
        const float2 q2{div2_ratio(make_float2(da, db), make_float2(na, nb))};
        if (__float_as_uint(q1.x) != __float_as_uint(__fdiv_rn(na, da)) ||
            __float_as_uint(q1.y) != __float_as_uint(__fdiv_rn(nb, db))) {
            atomicAdd(&bad[0], 1u);
        }
        if (__float_as_uint(q2.x) != __float_as_uint(__fdiv_rn(da, na)) ||
            __float_as_uint(q2.y) != __float_as_uint(__fdiv_rn(db, nb))) {
            atomicAdd(&bad[1], 1u);
        }
    }
}

int main() {
    unsigned int* d{nullptr};
    if (cudaMalloc(&d, 8) != cudaSuccess || cudaMemset(d, 0, 8) != cudaSuccess) return 2;
    const std::uint32_t lo{0u};            // +0
    const std::uint32_t hi{0x40800001u};   // just past 4.0f
    check<<<148 * 16, 256>>>(lo, hi, d);
    unsigned int h[2]{};
    if (cudaMemcpy(h, d, 8, cudaMemcpyDeviceToHost) != cudaSuccess) return 2;
    std::printf("floats %u: num/den mismatches %u, den/num mismatches %u\n", hi - lo, h[0], h[1]);
    cudaFree(d);
    return (h[0] | h[1]) != 0 ? 1 : 0;
}
