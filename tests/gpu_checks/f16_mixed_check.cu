// Check of the mixed-precision FP16-input instructions used by the frontend's
// chroma-from-luma sums (cujpegxl_b200/csrc/f16_mixed.cuh) against
// convert-then-FP32 arithmetic: every ordered pair (a, b) of finite FP16
// values, each with a pseudo-random finite float c (zero one time in eight),
// for fma_f16(a, b, c) == fmaf(float(a), float(b), c),
// add_f16(a, -float(b)) == float(a) - float(b) (the (b - y) form) and
// add_f16(a, c) == float(a) + c. Prints the mismatch counts; exits 1 on any.
#include <cstdint>
#include <cstdio>

#include "f16_mixed.cuh"

using namespace jxb;

__device__ std::uint32_t mix(std::uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__global__ void check(unsigned long long n, unsigned int* bad) {
    const unsigned long long stride{static_cast<unsigned long long>(gridDim.x) * blockDim.x};
    for (unsigned long long i{blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x}; i < n;
         i += stride) {
        const auto a{static_cast<unsigned short>(i & 0xffffu)};
        const auto b{static_cast<unsigned short>(i >> 16)};
        if (((a >> 10) & 31u) == 31u || ((b >> 10) & 31u) == 31u) continue;  // inf / nan
        const std::uint32_t h{mix(static_cast<std::uint32_t>(i))};
        float c{__uint_as_float((h & 0x807fffffu) | ((90u + (h >> 24) % 76u) << 23))};  // |c| in [2^-37, 2^38)
        if ((h & 7u) == 0u) c = 0.0f;
        const float fa{__half2float(__ushort_as_half(a))};
        const float fb{__half2float(__ushort_as_half(b))};
        if (__float_as_uint(fma_f16(a, b, c)) != __float_as_uint(__fmaf_rn(fa, fb, c))) atomicAdd(&bad[0], 1u);
        if (__float_as_uint(add_f16(a, -fb)) != __float_as_uint(__fadd_rn(fa, -fb))) atomicAdd(&bad[1], 1u);
        if (__float_as_uint(add_f16(a, c)) != __float_as_uint(__fadd_rn(fa, c))) atomicAdd(&bad[2], 1u);
    }
}

int main() {
    unsigned int* d{nullptr};
    if (cudaMalloc(&d, 12) != cudaSuccess || cudaMemset(d, 0, 12) != cudaSuccess) return 2;
    const unsigned long long n{1ull << 32};
    check<<<148 * 16, 256>>>(n, d);
    unsigned int h[3]{};
    if (cudaMemcpy(h, d, 12, cudaMemcpyDeviceToHost) != cudaSuccess) return 2;
    std::printf("operand pairs %llu: fma mismatches %u, sub mismatches %u, add mismatches %u\n", n, h[0], h[1], h[2]);
    cudaFree(d);
    return (h[0] | h[1] | h[2]) != 0 ? 1 : 0;
}
