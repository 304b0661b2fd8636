// Transform-decision network: inference inside an encode, and the training
// kernels (forward, backward-data, weight gradients, Adam) behind the C ABI.
//
// Every contraction is a BF16 x BF16 -> FP32 warp MMA (m16n8k16) fed by
// ldmatrix from shared memory. Convolutions are implicit GEMMs: the im2col
// row of an output position and eight consecutive reduction columns (one
// tap, eight input channels) is one 16-byte chunk of the [pixel][channel]
// activation buffer, or a zero chunk where the tap falls into the padding.
// The same chunk addressing serves the three products of training:
//   forward        Y[p][co]  = im2col(X)[p][k]  . W[co][k]^T
//   data gradient  dX[q][ci] = sum over (tap, co) of dY[p(q, tap)][co] . W[co][tap, ci]
//                  (a gather per input pixel, grouped by pixel parity for
//                  stride 2, so no scatter or atomics are needed)
//   weight grad.   dW[co][k] = dY[p][co]^T . im2col(X)[p][k]
// Reductions run in a fixed order, so training is deterministic.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "acsnet.cuh"
#include "cujpegxl/cujpegxl.h"
#include "cujpegxl_b200/cujpegxl_b200.h"
#include "frontend.cuh"
#include "jxl_constants.cuh"
#include "xyb.cuh"

namespace jxb {
namespace {

using bf16 = __nv_bfloat16;

constexpr int kNetThreads = 128;   // inference and training forward/backward CTAs
constexpr int kGradThreads = 256;  // weight-gradient CTAs
constexpr int kW1S = 88;           // shared-memory row stride of W1 (BF16)
constexpr int kWS = 296;           // row stride of W2..W4
constexpr int kActS = 40;          // pixel stride of 32-channel activations

// Weights and one region's activations. Row strides of 88/296/40 BF16 put the
// eight rows of every ldmatrix on distinct bank groups (stride-1 access).
struct NetWeights {
    bf16 w1[kNetC * kW1S];
    bf16 w[3][kNetC * kWS];
    float bias[4][kNetC];
    bf16 zero[8];
};

// Training: one region at a time.
struct NetSmem {
    NetWeights wt;
    bf16 x1[kNetInPix * kNetIn];
    bf16 x2[256 * kActS];
    bf16 x3[64 * kActS];
    bf16 x4[16 * kActS];
    float out[16 * kNetC];
};

struct TrainSmem {
    NetSmem n;
    bf16 g1[256 * kActS];
    bf16 g2[64 * kActS];
    bf16 g3[16 * kActS];
    bf16 g4[16 * kActS];
};

// Inference: the four regions of a 64x64 tile side by side, one warp group
// each. x1[r] holds the region's input (four channels per pixel, the first
// half of the buffer) and then its later activations (x3, x4 and the FP32
// outputs) once L1 has consumed it; x2 holds the tile's NV12 window until the
// inputs are built, then L1's output, then the partial sums of L3 and L4.
constexpr int kInferThreads = 512;
constexpr int kX3Off = 0;                          // BF16 offsets inside x1[r]
constexpr int kX4Off = kX3Off + 64 * kActS;
constexpr int kOutOff = kX4Off + 16 * kActS;       // FP32 [16][32] from here
constexpr int kInferX1 = kNetInPix * kNetIn;   // elements per region of x1
constexpr int kInferX2 = 256 * kActS;          // elements per region of x2
struct InferSmem {
    NetWeights wt;
    bf16 x1[4][kInferX1];
    bf16 x2[4][kInferX2];
};

static_assert(sizeof(NetWeights) % 16 == 0 && sizeof(NetSmem) % 16 == 0 && sizeof(TrainSmem) % 16 == 0,
              "16-byte shared-memory layout");
static_assert(2 * (kOutOff + 2 * 16 * kNetC) <= 2 * kNetInPix * kNetIn, "later activations exceed x1");
static_assert(sizeof(InferSmem) + 1024 <= 228 * 1024, "inference CTA too large");
static_assert(4 * 512 * sizeof(float) <= 256 * kActS * sizeof(bf16), "L3/L4 partial sums exceed x2");

__device__ __forceinline__ unsigned saddr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void ldsm_x4(unsigned (&r)[4], unsigned a) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a)
                 : "memory");
}

__device__ __forceinline__ void ldsm_x4_t(unsigned (&r)[4], unsigned a) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0, %1, %2, %3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(a)
                 : "memory");
}

__device__ __forceinline__ void ldsm_x2(unsigned (&r)[2], unsigned a) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0, %1}, [%2];\n"
                 : "=r"(r[0]), "=r"(r[1])
                 : "r"(a)
                 : "memory");
}

__device__ __forceinline__ void ldsm_x2_t(unsigned (&r)[2], unsigned a) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0, %1}, [%2];\n"
                 : "=r"(r[0]), "=r"(r[1])
                 : "r"(a)
                 : "memory");
}

// D += A . B for one 16x8x16 tile (A row-major 16x16, B column-major 16x8).
__device__ __forceinline__ void mma(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void store_pair(bf16* dst, float lo, float hi) {
    *reinterpret_cast<__nv_bfloat162*>(dst) = __floats2bfloat162_rn(lo, hi);
}

// Stored column of image column x in a row of width kW. With kPar the even
// columns come first, then the odd ones: the rows a stride-2 convolution
// gathers for consecutive outputs are then adjacent in memory, and the eight
// rows of an ldmatrix fall on distinct banks.
template <int kW, bool kPar>
__device__ __forceinline__ int par_col(int x) {
    return kPar ? (x & 1) * ((kW + 1) >> 1) + (x >> 1) : x;
}

// Shared-memory address of im2col row p, reduction columns k0..k0+7, for a
// 3x3 convolution with padding kPad over a kInW x kInW input of kCin channels
// stored kInS apart, kOutW x kOutW outputs; the zero chunk where the tap is
// padding (or a reduction column past the nine taps).
template <int kInW, int kOutW, int kStride, int kPad, int kCin, int kInS, bool kPar = false>
__device__ __forceinline__ unsigned im2col_row(unsigned in, unsigned zero, int p, int k0) {
    const int tap{k0 / kCin};
    const int ci{k0 - tap * kCin};
    const int oy{p / kOutW};
    const int ox{p - oy * kOutW};
    const int iy{oy * kStride + tap / 3 - kPad};
    const int ix{ox * kStride + tap % 3 - kPad};
    const bool ok{tap < 9 && iy >= 0 && iy < kInW && ix >= 0 && ix < kInW};
    return ok ? in + 2u * static_cast<unsigned>((iy * kInW + par_col<kInW, kPar>(ix)) * kInS + ci) : zero;
}

// im2col rows of one output position p, with everything that depends on p
// computed once: the address of the tap (0, 0) and a 9-bit mask of the taps
// inside the input. Tap (ky, kx) then lies a compile-time offset away: rows
// kInW apart, and columns at c(kx) from the position's column, where c is
// (kx - kPad) plainly and, in the parity-split layout (stride 2), the stored
// column of 2 ox + kx - kPad relative to ox.
template <int kInW, int kOutW, int kStride, int kPad, int kCin, int kInS, bool kPar = false>
struct Im2colRows {
    unsigned base;
    unsigned valid;

    __device__ __forceinline__ Im2colRows(unsigned in, int p) {
        const int oy{p / kOutW};
        const int ox{p - oy * kOutW};
        const int iy0{oy * kStride - kPad};
        const int ix0{ox * kStride - kPad};
        valid = 0;
#pragma unroll
        for (int t{0}; t < 9; ++t) {
            const int iy{iy0 + t / 3};
            const int ix{ix0 + t % 3};
            valid |= (iy >= 0 && iy < kInW && ix >= 0 && ix < kInW ? 1u : 0u) << t;
        }
        base = in + 2u * static_cast<unsigned>((iy0 * kInW + (kPar ? ox : ix0)) * kInS);
    }

    __host__ __device__ static constexpr int col(int kx) {
        return !kPar ? kx : ((((kx - kPad) & 1) != 0) ? (kInW + 1) / 2 + ((kx - kPad) >> 1) : ((kx - kPad) >> 1));
    }

    __host__ __device__ static constexpr unsigned offset(int tap, int ci) {
        return 2u * static_cast<unsigned>(((tap / 3) * kInW + col(tap % 3)) * kInS + ci);
    }

    __device__ __forceinline__ unsigned tap_at(unsigned zero, int tap, int ci) const {
        return tap < 9 && ((valid >> tap) & 1u) != 0 ? base + offset(tap, ci) : zero;
    }

    // Address of reduction columns k0 + 8h .. k0 + 8h + 7 (k0 a compile-time
    // constant once the caller's loop is unrolled, h the lane's half 0/1).
    __device__ __forceinline__ unsigned at(unsigned zero, int k0, int h) const {
        if (kCin >= 16) {  // both halves in one tap
            const int tap{k0 / kCin};
            return tap < 9 && ((valid >> tap) & 1u) != 0 ? base + offset(tap, k0 - tap * kCin) + 16u * h : zero;
        }
        return h ? tap_at(zero, k0 / kCin + 1, 0) : tap_at(zero, k0 / kCin, 0);
    }
};

// Forward of a layer with at least four 16-row position tiles (L1, L2): warp w
// takes position tiles w, w+4, ... (two at a time, 32 accumulators) and all
// four 8-channel output tiles.
template <int kInW, int kOutW, int kStride, int kPad, int kCin, int kInS, int kK, int kWStr, bool kParIn = false,
          bool kParOut = false>
__device__ __forceinline__ void fwd_rows(unsigned in, unsigned zero, unsigned w, const float* bias, bf16* out,
                                         int warp, int lane) {
    constexpr int kMW{kOutW * kOutW / 64};
    constexpr int kChunk{kMW < 2 ? kMW : 2};
    using Rows = Im2colRows<kInW, kOutW, kStride, kPad, kCin, kInS, kParIn>;
#pragma unroll 1
    for (int i0{0}; i0 < kMW; i0 += kChunk) {
        // kChunk is 1 or 2: the rows of position tiles i0 and i0 + kChunk - 1.
        const Rows rows0{in, (warp + 4 * i0) * 16 + (lane & 15)};
        const Rows rows1{in, (warp + 4 * (i0 + kChunk - 1)) * 16 + (lane & 15)};
        float acc[kChunk][4][4];
#pragma unroll
        for (int i{0}; i < kChunk; ++i) {
#pragma unroll
            for (int n{0}; n < 4; ++n) {
#pragma unroll
                for (int j{0}; j < 4; ++j) acc[i][n][j] = 0.0f;
            }
        }
        // Fully unrolled: every tap and channel offset is a compile-time constant.
#pragma unroll
        for (int k0{0}; k0 < kK; k0 += 16) {
            unsigned b[4][2];
#pragma unroll
            for (int h{0}; h < 2; ++h) {
                unsigned r[4];
                ldsm_x4(r, w + 2u * static_cast<unsigned>((h * 16 + (lane & 7) + ((lane >> 4) << 3)) * kWStr + k0 +
                                                          ((lane >> 3) & 1) * 8));
                b[2 * h][0] = r[0];
                b[2 * h][1] = r[1];
                b[2 * h + 1][0] = r[2];
                b[2 * h + 1][1] = r[3];
            }
#pragma unroll
            for (int i{0}; i < kChunk; ++i) {
                unsigned a[4];
                ldsm_x4(a, (i == 0 ? rows0 : rows1).at(zero, k0, lane >> 4));
#pragma unroll
                for (int n{0}; n < 4; ++n) mma(acc[i][n], a, b[n][0], b[n][1]);
            }
        }
#pragma unroll
        for (int i{0}; i < kChunk; ++i) {
            const int p{(warp + 4 * (i0 + i)) * 16 + (lane >> 2)};
            const int s0{(p / kOutW) * kOutW + par_col<kOutW, kParOut>(p % kOutW)};
            const int s1{((p + 8) / kOutW) * kOutW + par_col<kOutW, kParOut>((p + 8) % kOutW)};
#pragma unroll
            for (int n{0}; n < 4; ++n) {
                const int c{n * 8 + 2 * (lane & 3)};
                const float b0{bias[c]};
                const float b1{bias[c + 1]};
                store_pair(out + s0 * kActS + c, fmaxf(acc[i][n][0] + b0, 0.0f), fmaxf(acc[i][n][1] + b1, 0.0f));
                store_pair(out + s1 * kActS + c, fmaxf(acc[i][n][2] + b0, 0.0f), fmaxf(acc[i][n][3] + b1, 0.0f));
            }
        }
    }
}

// Forward of a layer with one 16-row position tile (L3, L4): warp w takes
// output channels 8w..8w+7. kRelu: BF16 activations; else FP32 outputs.
template <int kInW, int kStride, bool kRelu>
__device__ __forceinline__ void fwd_cols(unsigned in, unsigned zero, unsigned w, const float* bias, bf16* outb,
                                         float* outf, int warp, int lane) {
    // Two accumulators over alternate reduction steps halve the dependent
    // chain of tensor-core operations.
    float acc[2][4]{{0.0f, 0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f, 0.0f}};
    const Im2colRows<kInW, 4, kStride, 1, kNetC, kActS> rows{in, lane & 15};
#pragma unroll
    for (int k0{0}; k0 < kNetK; k0 += 16) {
        unsigned a[4];
        ldsm_x4(a, rows.at(zero, k0, lane >> 4));
        unsigned b[2];
        ldsm_x2(b, w + 2u * static_cast<unsigned>((8 * warp + (lane & 7)) * kWS + k0 + ((lane >> 3) & 1) * 8));
        mma(acc[(k0 >> 4) & 1], a, b[0], b[1]);
    }
    const int p{lane >> 2};
    const int c{8 * warp + 2 * (lane & 3)};
    const float v0{(acc[0][0] + acc[1][0]) + bias[c]};
    const float v1{(acc[0][1] + acc[1][1]) + bias[c + 1]};
    const float v2{(acc[0][2] + acc[1][2]) + bias[c]};
    const float v3{(acc[0][3] + acc[1][3]) + bias[c + 1]};
    if (kRelu) {
        store_pair(outb + p * kActS + c, fmaxf(v0, 0.0f), fmaxf(v1, 0.0f));
        store_pair(outb + (p + 8) * kActS + c, fmaxf(v2, 0.0f), fmaxf(v3, 0.0f));
    } else {
        outf[p * kNetC + c] = v0;
        outf[p * kNetC + c + 1] = v1;
        outf[(p + 8) * kNetC + c] = v2;
        outf[(p + 8) * kNetC + c + 1] = v3;
    }
}

// L2 of the inference for one position tile `mt` of two regions at once (the
// regions' L1 outputs in0 and in1, their L2 outputs out0 and out1): each
// weight fragment loaded serves both regions, which cuts the layer's
// shared-memory traffic by a third (its ldmatrix traffic bounds it); eight
// warps cover the tile's four regions.
__device__ __forceinline__ void fwd_l2_pair(unsigned in0, unsigned in1, unsigned zero, unsigned w, const float* bias,
                                            bf16* out0, bf16* out1, int mt, int lane) {
    using Rows = Im2colRows<16, 8, 2, 1, kNetC, kActS, true>;
    const Rows rows0{in0, mt * 16 + (lane & 15)};
    const Rows rows1{in1, mt * 16 + (lane & 15)};
    float acc[2][4][4];
#pragma unroll
    for (int i{0}; i < 2; ++i) {
#pragma unroll
        for (int n{0}; n < 4; ++n) {
#pragma unroll
            for (int j{0}; j < 4; ++j) acc[i][n][j] = 0.0f;
        }
    }
#pragma unroll
    for (int k0{0}; k0 < kNetK; k0 += 16) {
        unsigned b[4][2];
#pragma unroll
        for (int h{0}; h < 2; ++h) {
            unsigned r[4];
            ldsm_x4(r, w + 2u * static_cast<unsigned>((h * 16 + (lane & 7) + ((lane >> 4) << 3)) * kWS + k0 +
                                                      ((lane >> 3) & 1) * 8));
            b[2 * h][0] = r[0];
            b[2 * h][1] = r[1];
            b[2 * h + 1][0] = r[2];
            b[2 * h + 1][1] = r[3];
        }
#pragma unroll
        for (int i{0}; i < 2; ++i) {
            unsigned a[4];
            ldsm_x4(a, (i == 0 ? rows0 : rows1).at(zero, k0, lane >> 4));
#pragma unroll
            for (int n{0}; n < 4; ++n) mma(acc[i][n], a, b[n][0], b[n][1]);
        }
    }
    const int p{mt * 16 + (lane >> 2)};
#pragma unroll
    for (int i{0}; i < 2; ++i) {
        bf16* out{i == 0 ? out0 : out1};
#pragma unroll
        for (int n{0}; n < 4; ++n) {
            const int c{n * 8 + 2 * (lane & 3)};
            const float b0{bias[c]};
            const float b1{bias[c + 1]};
            store_pair(out + p * kActS + c, fmaxf(acc[i][n][0] + b0, 0.0f), fmaxf(acc[i][n][1] + b1, 0.0f));
            store_pair(out + (p + 8) * kActS + c, fmaxf(acc[i][n][2] + b0, 0.0f), fmaxf(acc[i][n][3] + b1, 0.0f));
        }
    }
}

// L3/L4 of the inference with the reduction split over the four warps of
// the region: warp kW takes reduction steps kS0 .. kS1 - 1 for all four
// output-channel tiles, stores its partial sums to `part`, and after a
// barrier every thread adds the four partials of its outputs in warp order.
template <int kInW, int kStride, int kS0, int kS1>
__device__ __forceinline__ void cols_partial(unsigned in, unsigned zero, unsigned w, float* part, int lane) {
    float acc[4][4]{};
    const Im2colRows<kInW, 4, kStride, 1, kNetC, kActS> rows{in, lane & 15};
#pragma unroll
    for (int s{kS0}; s < kS1; ++s) {
        const int k0{16 * s};
        unsigned a[4];
        ldsm_x4(a, rows.at(zero, k0, lane >> 4));
#pragma unroll
        for (int h{0}; h < 2; ++h) {
            unsigned r[4];
            ldsm_x4(r, w + 2u * static_cast<unsigned>((h * 16 + (lane & 7) + ((lane >> 4) << 3)) * kWS + k0 +
                                                      ((lane >> 3) & 1) * 8));
            mma(acc[2 * h], a, r[0], r[1]);
            mma(acc[2 * h + 1], a, r[2], r[3]);
        }
    }
    // part[(n * 4 + j) * 32 + lane]: fragment element j of channel tile n.
#pragma unroll
    for (int n{0}; n < 4; ++n) {
#pragma unroll
        for (int j{0}; j < 4; ++j) part[(n * 4 + j) * 32 + lane] = acc[n][j];
    }
}

template <int kInW, int kStride, bool kRelu>
__device__ __forceinline__ void fwd_cols_split(unsigned in, unsigned zero, unsigned w, const float* bias, bf16* outb,
                                               float* outf, float* part, int warp, int lane) {
    constexpr int kSteps{kNetK / 16};  // 18
    switch (warp) {
        case 0: cols_partial<kInW, kStride, 0, 5>(in, zero, w, part, lane); break;
        case 1: cols_partial<kInW, kStride, 5, 10>(in, zero, w, part + 512, lane); break;
        case 2: cols_partial<kInW, kStride, 10, 14>(in, zero, w, part + 1024, lane); break;
        default: cols_partial<kInW, kStride, 14, kSteps>(in, zero, w, part + 1536, lane); break;
    }
    __syncthreads();
    // Warp w finishes channel tile w: lane's fragment elements of tile w.
    const int n{warp};
    float v[4];
#pragma unroll
    for (int j{0}; j < 4; ++j) {
        const int at{(n * 4 + j) * 32 + lane};
        v[j] = ((part[at] + part[512 + at]) + part[1024 + at]) + part[1536 + at];
    }
    const int p{lane >> 2};
    const int c{8 * n + 2 * (lane & 3)};
    const float v0{v[0] + bias[c]};
    const float v1{v[1] + bias[c + 1]};
    const float v2{v[2] + bias[c]};
    const float v3{v[3] + bias[c + 1]};
    if (kRelu) {
        store_pair(outb + p * kActS + c, fmaxf(v0, 0.0f), fmaxf(v1, 0.0f));
        store_pair(outb + (p + 8) * kActS + c, fmaxf(v2, 0.0f), fmaxf(v3, 0.0f));
    } else {
        outf[p * kNetC + c] = v0;
        outf[p * kNetC + c + 1] = v1;
        outf[(p + 8) * kNetC + c] = v2;
        outf[(p + 8) * kNetC + c + 1] = v3;
    }
}

// Gradient into a BF16 buffer, zero where the layer input (post-ReLU) is zero.
__device__ __forceinline__ void store_masked(bf16* g, const bf16* x, int at, float v0, float v1) {
    const __nv_bfloat162 xv{*reinterpret_cast<const __nv_bfloat162*>(x + at)};
    const float m0{__bfloat162float(xv.x) > 0.0f ? v0 : 0.0f};
    const float m1{__bfloat162float(xv.y) > 0.0f ? v1 : 0.0f};
    store_pair(g + at, m0, m1);
}

// Data gradient of L4 (stride 1, 4x4): g3 = mask(x4) * convT(g4, W4). Warp w
// takes input channels 8w..8w+7 of the 16 pixels.
__device__ __forceinline__ void bwd_l4(unsigned gout, unsigned zero, unsigned w, const bf16* xin, bf16* gin,
                                       int warp, int lane) {
    float acc[4]{0.0f, 0.0f, 0.0f, 0.0f};
    const int q{lane & 15};
    const int qy{q >> 2};
    const int qx{q & 3};
#pragma unroll 2
    for (int s{0}; s < 18; ++s) {
        const int tap{s >> 1};
        const int co0{(s & 1) * 16};
        const int oy{qy - tap / 3 + 1};
        const int ox{qx - tap % 3 + 1};
        const bool ok{oy >= 0 && oy < 4 && ox >= 0 && ox < 4};
        unsigned a[4];
        ldsm_x4(a, ok ? gout + 2u * static_cast<unsigned>((oy * 4 + ox) * kActS + co0 + (lane >> 4) * 8) : zero);
        unsigned b[2];
        ldsm_x2_t(b, w + 2u * static_cast<unsigned>((co0 + (lane & 15)) * kWS + tap * kNetC + 8 * warp));
        mma(acc, a, b[0], b[1]);
    }
    const int p{lane >> 2};
    const int c{8 * warp + 2 * (lane & 3)};
    store_masked(gin, xin, p * kActS + c, acc[0], acc[1]);
    store_masked(gin, xin, (p + 8) * kActS + c, acc[2], acc[3]);
}

// Data gradient of a stride-2 layer over a kInW x kInW input. Input pixel
// (iy, ix) collects output position ((iy + 1 - ky) / 2, (ix + 1 - kx) / 2)
// for the taps whose offsets are even: ky = 1 for even iy, ky in {0, 2} for
// odd iy (the same in x). Pixels are processed in four parity classes, each
// a (kInW/2)^2 grid with its own tap list.
template <int kInW>
__device__ __forceinline__ void bwd_s2(unsigned gout, unsigned zero, unsigned w, const bf16* xin, bf16* gin,
                                       int warp, int lane) {
    constexpr int kOutW{kInW / 2};
    constexpr int kCW{kInW / 2};
    constexpr int kCM{kCW * kCW / 16};  // 16-pixel tiles per class
    static_assert(kCM == 1 || kCM == 4, "layer geometry");
#pragma unroll 1
    for (int cls{0}; cls < 4; ++cls) {
        const int py{cls >> 1};
        const int px{cls & 1};
        const int ntx{1 + px};
        const int nsteps{2 * (1 + py) * (1 + px)};
        // kCM == 4: warp w takes pixel tile w and all 32 channels; kCM == 1:
        // the single tile and channels 8w..8w+7.
        const int r{(kCM == 4 ? warp * 16 : 0) + (lane & 15)};
        const int iy{2 * (r / kCW) + py};
        const int ix{2 * (r % kCW) + px};
        float acc[4][4];
#pragma unroll
        for (int n{0}; n < 4; ++n) {
#pragma unroll
            for (int j{0}; j < 4; ++j) acc[n][j] = 0.0f;
        }
#pragma unroll 1
        for (int s{0}; s < nsteps; ++s) {
            const int j{s >> 1};
            const int co0{(s & 1) * 16};
            const int ky{py ? 2 * (j / ntx) : 1};
            const int kx{px ? 2 * (j % ntx) : 1};
            const int oy{(iy + 1 - ky) >> 1};
            const int ox{(ix + 1 - kx) >> 1};
            const bool ok{oy < kOutW && ox < kOutW};
            unsigned a[4];
            ldsm_x4(a, ok ? gout + 2u * static_cast<unsigned>((oy * kOutW + ox) * kActS + co0 + (lane >> 4) * 8)
                          : zero);
            const int col{(ky * 3 + kx) * kNetC};
            if (kCM == 4) {
#pragma unroll
                for (int h{0}; h < 2; ++h) {
                    unsigned bb[4];
                    ldsm_x4_t(bb, w + 2u * static_cast<unsigned>((co0 + (lane & 7) + ((lane >> 3) & 1) * 8) * kWS +
                                                                 col + h * 16 + (lane >> 4) * 8));
                    mma(acc[2 * h], a, bb[0], bb[1]);
                    mma(acc[2 * h + 1], a, bb[2], bb[3]);
                }
            } else {
                unsigned b[2];
                ldsm_x2_t(b, w + 2u * static_cast<unsigned>((co0 + (lane & 15)) * kWS + col + 8 * warp));
                mma(acc[0], a, b[0], b[1]);
            }
        }
        const int r0{(kCM == 4 ? warp * 16 : 0) + (lane >> 2)};
#pragma unroll
        for (int h{0}; h < 2; ++h) {
            const int rr{r0 + 8 * h};
            const int pix{(2 * (rr / kCW) + py) * kInW + 2 * (rr % kCW) + px};
            if (kCM == 4) {
#pragma unroll
                for (int n{0}; n < 4; ++n) {
                    store_masked(gin, xin, pix * kActS + n * 8 + 2 * (lane & 3), acc[n][2 * h], acc[n][2 * h + 1]);
                }
            } else {
                store_masked(gin, xin, pix * kActS + 8 * warp + 2 * (lane & 3), acc[0][2 * h], acc[0][2 * h + 1]);
            }
        }
    }
}

// Copies the weights into shared memory (rows padded to kW1S / kWS).
__device__ void load_net(NetWeights& s, const NetParamsDev& p, int tid, int nthreads) {
    const uint4* g{reinterpret_cast<const uint4*>(p.w)};
    for (int i{tid}; i < kNetC * (kNetK1 / 8); i += nthreads) {
        const int r{i / (kNetK1 / 8)};
        const int c{i - r * (kNetK1 / 8)};
        *reinterpret_cast<uint4*>(&s.w1[r * kW1S + c * 8]) = __ldg(&g[i]);
    }
    for (int l{0}; l < 3; ++l) {
        const uint4* gl{reinterpret_cast<const uint4*>(p.w + kNetW2 + l * kNetC * kNetK)};
        for (int i{tid}; i < kNetC * (kNetK / 8); i += nthreads) {
            const int r{i / (kNetK / 8)};
            const int c{i - r * (kNetK / 8)};
            *reinterpret_cast<uint4*>(&s.w[l][r * kWS + c * 8]) = __ldg(&gl[i]);
        }
    }
    for (int i{tid}; i < 4 * kNetC; i += nthreads) s.bias[i / kNetC][i % kNetC] = p.bias[i];
    if (tid < 8) s.zero[tid] = __float2bfloat16_rn(0.0f);
}

// One input pixel's eight stored channels: normalised X, Y, B and log2
// distance rounded to BF16, then four zeros.
__device__ __forceinline__ uint4 input_pixel(const NetParamsDev& p, float x, float y, float b, float l2d) {
    const float v0{(x - p.shift[0]) * p.scale[0]};
    const float v1{(y - p.shift[1]) * p.scale[1]};
    const float v2{(b - p.shift[2]) * p.scale[2]};
    const float v3{(l2d - p.shift[3]) * p.scale[3]};
    const __nv_bfloat162 lo{__floats2bfloat162_rn(v0, v1)};
    const __nv_bfloat162 hi{__floats2bfloat162_rn(v2, v3)};
    uint4 r;
    r.x = *reinterpret_cast<const unsigned*>(&lo);
    r.y = *reinterpret_cast<const unsigned*>(&hi);
    r.z = 0u;
    r.w = 0u;
    return r;
}

// L1 of the inference on inputs of four channels per pixel ([34][34][4]
// BF16, natural column order). Reduction step ky (16 columns) covers input
// row 2 oy + ky: its first eight columns are taps (ky, 0) and (ky, 1) (pixels
// 2 ox and 2 ox + 1, adjacent in memory), the next four tap (ky, 2) (pixel
// 2 ox + 2) and the last four pixel 2 ox + 3 against zero weights. Three
// steps instead of the five of the eight-channel layout (whose upper four
// channels and last eight columns are zeros), and an ldmatrix's eight rows
// (consecutive ox) are 16 contiguous bytes each.
constexpr int kL1PackedK = 48;
__device__ __forceinline__ void pack_w1(NetWeights& s, const NetParamsDev& p, int tid, int nthreads) {
    for (int i{tid}; i < kNetC * kL1PackedK; i += nthreads) {
        const int co{i / kL1PackedK};
        const int k{i - co * kL1PackedK};
        const int ky{k >> 4};
        const int j{k & 15};
        std::uint16_t v{0};
        if (j < 12) {
            const int tap{3 * ky + (j < 8 ? j >> 2 : 2)};
            v = p.w[kNetW1 + co * kNetK1 + tap * kNetIn + (j & 3)];
        }
        reinterpret_cast<std::uint16_t*>(s.w1)[co * kW1S + k] = v;
    }
}

__device__ __forceinline__ void fwd_l1_packed(unsigned in, unsigned w, const float* bias, bf16* out, int warp,
                                              int lane) {
#pragma unroll 1
    for (int i0{0}; i0 < 4; i0 += 2) {
        unsigned base[2];
#pragma unroll
        for (int i{0}; i < 2; ++i) {
            const int pos{(warp + 4 * (i0 + i)) * 16 + (lane & 15)};
            const int oy{pos >> 4};
            const int ox{pos & 15};
            base[i] = in + 2u * static_cast<unsigned>((2 * oy * kNetInW + 2 * ox) * 4) + 16u * (lane >> 4);
        }
        float acc[2][4][4];
#pragma unroll
        for (int i{0}; i < 2; ++i) {
#pragma unroll
            for (int n{0}; n < 4; ++n) {
#pragma unroll
                for (int j{0}; j < 4; ++j) acc[i][n][j] = 0.0f;
            }
        }
#pragma unroll
        for (int ky{0}; ky < 3; ++ky) {
            unsigned b[4][2];
#pragma unroll
            for (int h{0}; h < 2; ++h) {
                unsigned r[4];
                ldsm_x4(r, w + 2u * static_cast<unsigned>((h * 16 + (lane & 7) + ((lane >> 4) << 3)) * kW1S + 16 * ky +
                                                          ((lane >> 3) & 1) * 8));
                b[2 * h][0] = r[0];
                b[2 * h][1] = r[1];
                b[2 * h + 1][0] = r[2];
                b[2 * h + 1][1] = r[3];
            }
#pragma unroll
            for (int i{0}; i < 2; ++i) {
                unsigned a[4];
                ldsm_x4(a, base[i] + 2u * static_cast<unsigned>(ky * kNetInW * 4));
#pragma unroll
                for (int n{0}; n < 4; ++n) mma(acc[i][n], a, b[n][0], b[n][1]);
            }
        }
#pragma unroll
        for (int i{0}; i < 2; ++i) {
            const int p{(warp + 4 * (i0 + i)) * 16 + (lane >> 2)};
            const int s0{(p / 16) * 16 + par_col<16, true>(p % 16)};
            const int s1{((p + 8) / 16) * 16 + par_col<16, true>((p + 8) % 16)};
#pragma unroll
            for (int n{0}; n < 4; ++n) {
                const int c{n * 8 + 2 * (lane & 3)};
                const float b0{bias[c]};
                const float b1{bias[c + 1]};
                store_pair(out + s0 * kActS + c, fmaxf(acc[i][n][0] + b0, 0.0f), fmaxf(acc[i][n][1] + b1, 0.0f));
                store_pair(out + s1 * kActS + c, fmaxf(acc[i][n][2] + b0, 0.0f), fmaxf(acc[i][n][3] + b1, 0.0f));
            }
        }
    }
}

// The four layers over the region in s.x1; ends with s.out filled.
// warp: the warp's index (0..3) within the group of four warps that owns the
// region; every thread of the CTA calls this together.
// kInfer: the inference layout and schedule: x1 holds four channels per
// pixel in natural column order (L1 by fwd_l1_packed), x2 is stored with its
// columns parity-split (par_col), and L3 and L4 split their reduction over
// the group's warps with x2 as the scratch of their partial sums. Otherwise
// (training) x1 holds eight channels per pixel and nothing is parity-split.
template <bool kInfer = false>
__device__ __forceinline__ void net_forward(const NetWeights& wt, bf16* x1, bf16* x2, bf16* x3, bf16* x4,
                                            float* out, int warp, int lane, int grp = 0) {
    const unsigned zero{saddr(wt.zero)};
    if constexpr (kInfer) {
        fwd_l1_packed(saddr(x1), saddr(wt.w1), wt.bias[0], x2, warp, lane);
    } else {
        fwd_rows<kNetInW, 16, 2, 0, kNetIn, kNetIn, kNetK1, kW1S, kInfer, kInfer>(saddr(x1), zero, saddr(wt.w1),
                                                                            wt.bias[0], x2, warp, lane);
    }
    __syncthreads();
    if constexpr (kInfer) {
        // Groups 0 and 1 take regions (0, 1) and (2, 3); the four regions'
        // buffers lie kInferX1 / kInferX2 elements apart.
        if (grp < 2) {
            const int r0{2 * grp};
            bf16* x2r0{x2 + (r0 - grp) * kInferX2};
            bf16* x1r0{x1 + (r0 - grp) * kInferX1};
            fwd_l2_pair(saddr(x2r0), saddr(x2r0 + kInferX2), zero, saddr(wt.w[0]), wt.bias[1], x1r0 + kX3Off,
                        x1r0 + kInferX1 + kX3Off, warp, lane);
        }
    } else {
        fwd_rows<16, 8, 2, 1, kNetC, kActS, kNetK, kWS, kInfer, false>(saddr(x2), zero, saddr(wt.w[0]), wt.bias[1],
                                                                     x3, warp, lane);
    }
    __syncthreads();
    if constexpr (kInfer) {
        fwd_cols_split<8, 2, true>(saddr(x3), zero, saddr(wt.w[1]), wt.bias[2], x4, nullptr,
                                   reinterpret_cast<float*>(x2), warp, lane);
    } else {
        fwd_cols<8, 2, true>(saddr(x3), zero, saddr(wt.w[1]), wt.bias[2], x4, nullptr, warp, lane);
    }
    __syncthreads();
    if constexpr (kInfer) {
        fwd_cols_split<4, 1, false>(saddr(x4), zero, saddr(wt.w[2]), wt.bias[3], nullptr, out,
                                    reinterpret_cast<float*>(x2), warp, lane);
    } else {
        fwd_cols<4, 1, false>(saddr(x4), zero, saddr(wt.w[2]), wt.bias[3], nullptr, out, warp, lane);
    }
    __syncthreads();
}

// Split logit of `lane` (0..16; -inf elsewhere): channel 1 + lane averaged
// over the 16 positions, summed in position order.
__device__ __forceinline__ float split_logit(const float* out, int lane) {
    if (lane >= kNetClasses) return -INFINITY;
    float acc{0.0f};
#pragma unroll
    for (int p{0}; p < 16; ++p) acc = acc + out[p * kNetC + 1 + lane];
    return acc * 0.0625f;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o{16}; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o{16}; o > 0; o >>= 1) v = v + __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Lowest lane holding the warp maximum of v.
__device__ __forceinline__ int warp_argmax(float v, float mx) {
    return __ffs(__ballot_sync(0xffffffffu, v == mx)) - 1;
}

// Softmax statistics of the split logits held one per lane.
struct SplitHead {
    float prob;    // this lane's probability
    int top;       // arg-max class
    float margin;  // top probability minus the runner-up
    float lse;     // log-sum-exp of the logits
};

__device__ __forceinline__ SplitHead split_head(float logit) {
    const int lane{static_cast<int>(threadIdx.x & 31)};
    const float mx{warp_max(logit)};
    const float e{logit == -INFINITY ? 0.0f : expf(logit - mx)};
    const float sum{warp_sum(e)};
    SplitHead h;
    h.prob = e / sum;
    h.top = warp_argmax(logit, mx);
    const float second{warp_max(lane == h.top ? 0.0f : e)};
    h.margin = (__shfl_sync(0xffffffffu, e, h.top) - second) / sum;
    h.lse = logf(sum) + mx;
    return h;
}

// ---- Inference inside an encode ----

// Hardware base-2 exponential and logarithm (PTX ex2/lg2.approx), in their
// flush-to-zero forms, which are one instruction each (the forms that keep
// subnormals add a range check and scaling around it). Every argument and
// result below is a normal float (logarithms of values >= 0.0037, powers
// between 2^-9 and 2), so flushing changes no value; it took the network's
// input stage from 14.4K to 8.6K cycles per 64x64 tile.
__device__ __forceinline__ float hw_exp2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float hw_log2(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// The network's input pixels: xyb_pixel's NV12 -> XYB conversion of two
// pixels at once (component h of every result is pixel h), from each pixel's
// luma byte and its four chroma taps ((cb, cr) pairs as 16-bit words:
// top-left, top-right, bottom-left, bottom-right, weights wxa (left) and
// wya (top) in {1, 3}), with the two transfer functions taken from the
// hardware exp2/log2 (x^2.4 = 2^(2.4 log2 x), cbrt x = 2^(log2 x / 3))
// instead of the frontend's exact ones. The values differ from the
// frontend's by about 1e-6 relative, far below the BF16 rounding of the
// input (4e-3), at a fraction of the instructions. The arithmetic runs on
// packed f32x2 pairs (each component rounded as the scalar operation); the
// transfer functions stay scalar.
__device__ __forceinline__ void net_xyb_taps2(const int (&luma)[2], const unsigned (&aa)[2], const unsigned (&ab)[2],
                                              const unsigned (&ba)[2], const unsigned (&bb)[2], int wxa,
                                              const int (&wya)[2], float2& ox, float2& oy, float2& ob) {
    const float2 yv{__fmul2_rn(make_float2(static_cast<float>(luma[0]), static_cast<float>(luma[1])), f2dup(kInv255))};
    const int wxb{4 - wxa};
    int scb[2], scr[2];
#pragma unroll
    for (int h{0}; h < 2; ++h) {
        const int wyb{4 - wya[h]};
        scb[h] = wya[h] * (wxa * static_cast<int>(aa[h] & 0xffu) + wxb * static_cast<int>(ab[h] & 0xffu)) +
                 wyb * (wxa * static_cast<int>(ba[h] & 0xffu) + wxb * static_cast<int>(bb[h] & 0xffu));
        scr[h] = wya[h] * (wxa * static_cast<int>(aa[h] >> 8) + wxb * static_cast<int>(ab[h] >> 8)) +
                 wyb * (wxa * static_cast<int>(ba[h] >> 8) + wxb * static_cast<int>(bb[h] >> 8));
    }
    const float2 cb{__fadd2_rn(__fmul2_rn(make_float2(static_cast<float>(scb[0]), static_cast<float>(scb[1])),
                                          f2dup(1.0f / 4080.0f)),
                               f2dup(-kChromaCenter))};
    const float2 cr{__fadd2_rn(__fmul2_rn(make_float2(static_cast<float>(scr[0]), static_cast<float>(scr[1])),
                                          f2dup(1.0f / 4080.0f)),
                               f2dup(-kChromaCenter))};
    auto lin = [](float2 e) {
        e = clamp01_2(e);
        const float2 lo{__fmul2_rn(e, f2dup(1.0f / 12.92f))};
        const float2 t{__fmul2_rn(__fadd2_rn(e, f2dup(0.055f)), f2dup(1.0f / 1.055f))};
        const float2 l{__fmul2_rn(f2dup(2.4f), make_float2(hw_log2(t.x), hw_log2(t.y)))};
        const float2 hi{hw_exp2(l.x), hw_exp2(l.y)};
        return clamp01_2(make_float2(e.x <= 0.04045f ? lo.x : hi.x, e.y <= 0.04045f ? lo.y : hi.y));
    };
    const float2 r{lin(__ffma2_rn(f2dup(kCrToR), cr, yv))};
    const float2 g{lin(__ffma2_rn(f2dup(-kCrToG), cr, __ffma2_rn(f2dup(-kCbToG), cb, yv)))};
    const float2 b{lin(__ffma2_rn(f2dup(kCbToB), cb, yv))};
    auto cbrt_pos = [](float2 v) {
        const float2 l{__fmul2_rn(make_float2(hw_log2(v.x), hw_log2(v.y)), f2dup(1.0f / 3.0f))};
        return make_float2(v.x > 0.0f ? hw_exp2(l.x) : 0.0f, v.y > 0.0f ? hw_exp2(l.y) : 0.0f);
    };
    const float2 bias{f2dup(kOpsinBias)};
    const float2 nb{f2dup(kNegCbrtBias)};
    const float2 m0{__fadd2_rn(
        cbrt_pos(__ffma2_rn(f2dup(kM02), b, __ffma2_rn(f2dup(kM01), g, __ffma2_rn(f2dup(kM00), r, bias)))), nb)};
    const float2 m1{__fadd2_rn(
        cbrt_pos(__ffma2_rn(f2dup(kM12), b, __ffma2_rn(f2dup(kM11), g, __ffma2_rn(f2dup(kM10), r, bias)))), nb)};
    const float2 m2{__fadd2_rn(
        cbrt_pos(__ffma2_rn(f2dup(kM22), b, __ffma2_rn(f2dup(kM21), g, __ffma2_rn(f2dup(kM20), r, bias)))), nb)};
    ox = __fmul2_rn(f2dup(0.5f), __fadd2_rn(m0, f2neg(m1)));
    oy = __fmul2_rn(f2dup(0.5f), __fadd2_rn(m0, m1));
    ob = m2;
}

constexpr int kTileWin = kNetInW + 32;     // luma window of a 64x64 tile and its 1-pixel ring
constexpr int kTileChroma = 32 + 4;        // chroma window of the tile (2-sample margins)

// One CTA per SM walks the frame's 64x64 tiles; its four warp groups each
// take one of the tile's four regions through the network in lockstep (one
// barrier per layer for all four). The weights are loaded once per CTA.
__global__ void __launch_bounds__(kInferThreads, 1)
    acsnet_infer_kernel(FrontendInputs in, NetParamsDev p, float log2_distance, float margin,
                        NetDecisionsDev out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    InferSmem& s{*reinterpret_cast<InferSmem*>(smem_raw)};
    const int tid{static_cast<int>(threadIdx.x)};
    const int warp{tid >> 5};
    const int lane{tid & 31};
    const int grp{warp >> 2};
    // Set when a region of the current tile inside the image is left to the
    // heuristic (its tile goes to the back of out.tile_order).
    __shared__ unsigned sh_heuristic;
    if (tid == 0) sh_heuristic = 0;
    load_net(s.wt, p, tid, kInferThreads);
    __syncthreads();
    pack_w1(s.wt, p, tid, kInferThreads);
    const int W{in.width};
    const int H{in.height};
    const int bw{W >> 3};
    const int rw{(bw + 3) >> 2};
    const int rh{((H >> 3) + 3) >> 2};
    const int tw{(W + 63) >> 6};
    const int ntiles{tw * ((H + 63) >> 6)};
    std::uint8_t* win_luma{reinterpret_cast<std::uint8_t*>(s.x2)};
    std::uint8_t* win_chroma{win_luma + kTileWin * kTileWin + 4};
    bf16* x1{s.x1[grp]};
    float* o{reinterpret_cast<float*>(x1 + kOutOff)};
    // The NV12 window of the next tile is loaded into registers while the
    // current one runs through the network, then stored to shared memory.
    constexpr int kLumaPer{(kTileWin * kTileWin + kInferThreads - 1) / kInferThreads};
    constexpr int kChromaPer{(kTileChroma * kTileChroma + kInferThreads - 1) / kInferThreads};
    unsigned pl[kLumaPer];
    unsigned pc[kChromaPer];
    auto fetch = [&](int t) {
        const int px0{(t % tw) * 64};
        const int py0{(t / tw) * 64};
        const int cx0{(px0 >> 1) - 2};
        const int cy0{(py0 >> 1) - 2};
#pragma unroll
        for (int j{0}; j < kLumaPer; ++j) {
            const int i{tid + j * kInferThreads};
            if (i < kTileWin * kTileWin) {
                const int gx{min(max(px0 - 1 + i % kTileWin, 0), W - 1)};
                const int gy{min(max(py0 - 1 + i / kTileWin, 0), H - 1)};
                pl[j] = __ldg(in.luma + static_cast<std::size_t>(gy) * in.luma_pitch + gx);
            }
        }
#pragma unroll
        for (int j{0}; j < kChromaPer; ++j) {
            const int i{tid + j * kInferThreads};
            if (i < kTileChroma * kTileChroma) {
                const int jx{min(max(cx0 + i % kTileChroma, 0), (W >> 1) - 1)};
                const int jy{min(max(cy0 + i / kTileChroma, 0), (H >> 1) - 1)};
                const std::uint8_t* c{in.chroma + static_cast<std::size_t>(jy) * in.chroma_pitch + 2 * jx};
                pc[j] = __ldg(c) | (static_cast<unsigned>(__ldg(c + 1)) << 8);
            }
        }
    };
    if (static_cast<int>(blockIdx.x) < ntiles) fetch(static_cast<int>(blockIdx.x));
    for (int t{static_cast<int>(blockIdx.x)}; t < ntiles; t += static_cast<int>(gridDim.x)) {
        const int px0{(t % tw) * 64};
        const int py0{(t / tw) * 64};
        unsigned full{0};  // regions of the tile that are a full 32x32 inside the image
#pragma unroll
        for (int r{0}; r < 4; ++r) {
            full |= (px0 + 32 * (r & 1) + 32 <= W && py0 + 32 * (r >> 1) + 32 <= H ? 1u : 0u) << r;
        }
        __syncthreads();  // the previous tile is done with the window and the outputs
#pragma unroll
        for (int j{0}; j < kLumaPer; ++j) {
            const int i{tid + j * kInferThreads};
            if (i < kTileWin * kTileWin) win_luma[i] = static_cast<std::uint8_t>(pl[j]);
        }
#pragma unroll
        for (int j{0}; j < kChromaPer; ++j) {
            const int i{tid + j * kInferThreads};
            if (i < kTileChroma * kTileChroma) {
                win_chroma[2 * i] = static_cast<std::uint8_t>(pc[j]);
                win_chroma[2 * i + 1] = static_cast<std::uint8_t>(pc[j] >> 8);
            }
        }
        __syncthreads();
        if (t + static_cast<int>(gridDim.x) < ntiles) fetch(t + static_cast<int>(gridDim.x));
        if (full != 0) {   // block-uniform
            const int cx0{(px0 >> 1) - 2};
            const int cy0{(py0 >> 1) - 2};
            // Thread t takes column t % 34 of rows t / 34, t / 34 + 15, ...
            // of the regions, rows row (region rx) and 32 + row (region
            // 2 + rx) as one pixel pair: its column's chroma taps and clamps
            // are computed once, and a warp's stores are contiguous.
            constexpr int kRowLanes{kInferThreads / kNetInW};  // 15
            if (tid < kNetInW * kRowLanes) {
                const int x{tid % kNetInW};
                const auto* cw{reinterpret_cast<const std::uint16_t*>(win_chroma)};
#pragma unroll
                for (int rx{0}; rx < 2; ++rx) {
                    const int wx{32 * rx + x};
                    const int gx{min(max(px0 - 1 + wx, 0), W - 1)};
                    const int jx{gx >> 1};
                    const int xa{((gx & 1) ? jx : max(jx - 1, 0)) - cx0};
                    const int xb{((gx & 1) ? min(jx + 1, (W >> 1) - 1) : jx) - cx0};
                    const int wxa{(gx & 1) ? 3 : 1};
                    // Rows row (region rx) and 32 + row (region 2 + rx) as one pair.
                    const bool top{((full >> rx) & 1u) != 0};
                    const bool bot{((full >> (2 + rx)) & 1u) != 0};
                    if (!top && !bot) continue;
#pragma unroll
                    for (int row{tid / kNetInW}; row < kNetInW; row += kRowLanes) {
                        int luma[2], wya[2];
                        unsigned aa[2], ab[2], ba[2], bb[2];
#pragma unroll
                        for (int h{0}; h < 2; ++h) {
                            const int wy{32 * h + row};
                            const int gy{min(max(py0 - 1 + wy, 0), H - 1)};
                            const int jy{gy >> 1};
                            const int ya{(((gy & 1) ? jy : max(jy - 1, 0)) - cy0) * kTileChroma};
                            const int yb{(((gy & 1) ? min(jy + 1, (H >> 1) - 1) : jy) - cy0) * kTileChroma};
                            luma[h] = win_luma[wy * kTileWin + wx];
                            aa[h] = cw[ya + xa];
                            ab[h] = cw[ya + xb];
                            ba[h] = cw[yb + xa];
                            bb[h] = cw[yb + xb];
                            wya[h] = (gy & 1) ? 3 : 1;
                        }
                        float2 xv, yv, bv;
                        net_xyb_taps2(luma, aa, ab, ba, bb, wxa, wya, xv, yv, bv);
                        const float2 nx{__fmul2_rn(__fadd2_rn(xv, f2dup(-p.shift[0])), f2dup(p.scale[0]))};
                        const float2 ny{__fmul2_rn(__fadd2_rn(yv, f2dup(-p.shift[1])), f2dup(p.scale[1]))};
                        const float2 nbv{__fmul2_rn(__fadd2_rn(bv, f2dup(-p.shift[2])), f2dup(p.scale[2]))};
                        const float nd{(log2_distance - p.shift[3]) * p.scale[3]};
                        const int at{(row * kNetInW + x) * 4};
                        if (top) {
                            const __nv_bfloat162 lo{__floats2bfloat162_rn(nx.x, ny.x)};
                            const __nv_bfloat162 hi{__floats2bfloat162_rn(nbv.x, nd)};
                            *reinterpret_cast<uint2*>(&s.x1[rx][at]) =
                                make_uint2(*reinterpret_cast<const unsigned*>(&lo), *reinterpret_cast<const unsigned*>(&hi));
                        }
                        if (bot) {
                            const __nv_bfloat162 lo{__floats2bfloat162_rn(nx.y, ny.y)};
                            const __nv_bfloat162 hi{__floats2bfloat162_rn(nbv.y, nd)};
                            *reinterpret_cast<uint2*>(&s.x1[2 + rx][at]) =
                                make_uint2(*reinterpret_cast<const unsigned*>(&lo), *reinterpret_cast<const unsigned*>(&hi));
                        }
                    }
                }
            }
            __syncthreads();
            // Groups of regions outside the image run on stale data and
            // their results are dropped.
            net_forward<true>(s.wt, x1, s.x2[grp], x1 + kX3Off, x1 + kX4Off, o, warp & 3, lane, grp);
        }
        if ((warp & 3) == 0) {
            const int rx{2 * (t % tw) + (grp & 1)};
            const int ry{2 * (t / tw) + (grp >> 1)};
            if (rx < rw && ry < rh) {
                int cls{-1};
                if (((full >> grp) & 1u) != 0) {
                    const SplitHead h{split_head(split_logit(o, lane))};
                    cls = h.margin >= margin ? h.top : -1;
                }
                if (lane == 0) {
                    out.cls[ry * rw + rx] = static_cast<std::int8_t>(cls);
                    if (cls < 0) atomicOr(&sh_heuristic, 1u);
                }
                if (cls >= 0 && out.qf != nullptr && lane < 16) {
                    // fmaxf maps a NaN to 1.
                    const float q{fminf(fmaxf(rintf(exp2f(o[lane * kNetC])), 1.0f), static_cast<float>(kQuantMax))};
                    out.qf[static_cast<std::size_t>(ry * 4 + (lane >> 2)) * bw + rx * 4 + (lane & 3)] =
                        static_cast<std::int16_t>(static_cast<int>(q));
                }
            }
        }
        if (out.tile_order != nullptr) {  // the same for every thread
            __syncthreads();  // every region's flag is in
            if (tid == 0) {
                const unsigned n{static_cast<unsigned>(ntiles)};
                const unsigned at{sh_heuristic == 0 ? atomicAdd(&out.tile_order[n], 1u)
                                                    : n - 1u - atomicAdd(&out.tile_order[n + 1], 1u)};
                out.tile_order[at] = static_cast<std::uint32_t>(t);
                sh_heuristic = 0;
            }
        }
    }
}

// ---- Training ----

// Forward (and with labels the loss and the data gradients) of one sample per
// iteration; stores the activations and gradients the weight-gradient kernel
// needs. out[n][33] and stats[n][4] are optional.
__global__ void __launch_bounds__(kNetThreads)
    acsnet_train_kernel(NetParamsDev p, NetBatchDev b, float inv_batch, float qf_weight, bf16* act,
                        float* outv, float* stats) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainSmem& ts{*reinterpret_cast<TrainSmem*>(smem_raw)};
    NetSmem& s{ts.n};
    const int tid{static_cast<int>(threadIdx.x)};
    const int warp{tid >> 5};
    const int lane{tid & 31};
    load_net(s.wt, p, tid, kNetThreads);
    const unsigned zero{saddr(s.wt.zero)};
    for (std::uint32_t i{blockIdx.x}; i < b.n; i += gridDim.x) {
        __syncthreads();
        const float* tile{b.tiles + static_cast<std::size_t>(b.tile_index[i]) * 3 * kNetInPix};
        const float l2d{b.log2_distance[i]};
        for (int px{tid}; px < kNetInPix; px += kNetThreads) {
            *reinterpret_cast<uint4*>(&s.x1[px * kNetIn]) =
                input_pixel(p, tile[px], tile[kNetInPix + px], tile[2 * kNetInPix + px], l2d);
        }
        __syncthreads();
        net_forward(s.wt, s.x1, s.x2, s.x3, s.x4, s.out, warp, lane);
        if (outv != nullptr && warp == 0) {
            float* o{outv + static_cast<std::size_t>(i) * kNetOut};
            const float lg{split_logit(s.out, lane)};
            if (lane < kNetClasses) o[lane] = lg;
            if (lane < 16) o[kNetClasses + lane] = s.out[lane * kNetC];
        }
        if (b.label_class == nullptr) continue;  // block-uniform
        if (warp == 0) {
            // Loss and its gradient at the L4 outputs.
            const int label{b.label_class[i]};
            const float lg{split_logit(s.out, lane)};
            const SplitHead h{split_head(lg)};
            // Target: the label's one-hot vector, or a given distribution.
            float t{lane == label ? 1.0f : 0.0f};
            if (b.label_soft != nullptr) {
                t = lane < kNetClasses ? b.label_soft[static_cast<std::size_t>(i) * kNetClasses + lane] : 0.0f;
            }
            const float dlogit{(h.prob - t) * inv_batch};
            const float ce{h.lse - warp_sum(lane < kNetClasses ? t * lg : 0.0f)};
            float d{0.0f};
            if (lane < 16) d = s.out[lane * kNetC] - b.label_qf[static_cast<std::size_t>(i) * 16 + lane];
            const float sq{warp_sum(d * d)};
            const float dq{2.0f * qf_weight * d * inv_batch * 0.0625f};
            const float dl_c{__shfl_sync(0xffffffffu, dlogit, (lane + 31) & 31) * 0.0625f};
#pragma unroll 1
            for (int pp{0}; pp < 16; ++pp) {
                const float dqp{__shfl_sync(0xffffffffu, dq, pp)};
                const float v{lane == 0 ? dqp : (lane <= kNetClasses ? dl_c : 0.0f)};
                ts.g4[pp * kActS + lane] = __float2bfloat16_rn(v);
            }
            if (stats != nullptr && lane == 0) {
                float* st{stats + static_cast<std::size_t>(i) * 4};
                st[0] = ce;
                st[1] = sq * 0.0625f;
                st[2] = h.top == label ? 1.0f : 0.0f;
                st[3] = h.margin;
            }
        }
        __syncthreads();
        bwd_l4(saddr(ts.g4), zero, saddr(s.wt.w[2]), s.x4, ts.g3, warp, lane);
        __syncthreads();
        bwd_s2<8>(saddr(ts.g3), zero, saddr(s.wt.w[1]), s.x3, ts.g2, warp, lane);
        __syncthreads();
        bwd_s2<16>(saddr(ts.g2), zero, saddr(s.wt.w[0]), s.x2, ts.g1, warp, lane);
        __syncthreads();
        // Compact copies for the weight-gradient kernel (8 BF16 per uint4).
        bf16* a{act + static_cast<std::size_t>(i) * kNetActPerSample};
        auto put = [&](int dst, const bf16* src, int pixels, int stride, int ch) {
            const int per{ch / 8};
            for (int k{tid}; k < pixels * per; k += kNetThreads) {
                const int px{k / per};
                const int c{k - px * per};
                *reinterpret_cast<uint4*>(a + dst + px * ch + c * 8) =
                    *reinterpret_cast<const uint4*>(src + px * stride + c * 8);
            }
        };
        put(kNetActX1, s.x1, kNetInPix, kNetIn, kNetIn);
        put(kNetActX2, s.x2, 256, kActS, kNetC);
        put(kNetActX3, s.x3, 64, kActS, kNetC);
        put(kNetActX4, s.x4, 16, kActS, kNetC);
        put(kNetActG1, ts.g1, 256, kActS, kNetC);
        put(kNetActG2, ts.g2, 64, kActS, kNetC);
        put(kNetActG3, ts.g3, 16, kActS, kNetC);
        put(kNetActG4, ts.g4, 16, kActS, kNetC);
    }
}

// Geometry of layer L (1..4) for the weight gradient.
template <int L>
struct LayerGeo {
    static constexpr int kInW = L == 1 ? kNetInW : (L == 2 ? 16 : (L == 3 ? 8 : 4));
    static constexpr int kOutW = L == 1 ? 16 : (L == 2 ? 8 : 4);
    static constexpr int kPad = L == 1 ? 0 : 1;
    static constexpr int kStride = L == 4 ? 1 : 2;
    static constexpr int kCin = L == 1 ? kNetIn : kNetC;
    static constexpr int kInS = L == 1 ? kNetIn : kActS;
    static constexpr int kK = L == 1 ? kNetK1 : kNetK;
    static constexpr int kP = kOutW * kOutW;
    static constexpr int kXOff = L == 1 ? kNetActX1 : (L == 2 ? kNetActX2 : (L == 3 ? kNetActX3 : kNetActX4));
    static constexpr int kGOff = L == 1 ? kNetActG1 : (L == 2 ? kNetActG2 : (L == 3 ? kNetActG3 : kNetActG4));
    static constexpr int kWOff = L == 1 ? kNetW1 : (L == 2 ? kNetW2 : (L == 3 ? kNetW3 : kNetW4));
};

// dW_L = sum over the split's samples and positions of g[p][co] x im2col(x)[p][k],
// and the bias gradient; written to partial[blockIdx.x][...] in fixed order.
template <int L>
__global__ void __launch_bounds__(kGradThreads) acsnet_wgrad_kernel(const bf16* act, std::uint32_t n, float* partial) {
    using G = LayerGeo<L>;
    constexpr int kPairs{G::kK / 16};   // pairs of 8-column tiles
    constexpr int kPW{(kPairs + 7) / 8};  // pairs per warp
    __shared__ __align__(16) bf16 xs[G::kInW * G::kInW * G::kInS];
    __shared__ __align__(16) bf16 gs[G::kP * kActS];
    __shared__ __align__(16) bf16 zs[8];
    const int tid{static_cast<int>(threadIdx.x)};
    const int warp{tid >> 5};
    const int lane{tid & 31};
    if (tid < 8) zs[tid] = __float2bfloat16_rn(0.0f);
    float acc[kPW][2][2][4];
#pragma unroll
    for (int i{0}; i < kPW; ++i) {
#pragma unroll
        for (int m{0}; m < 2; ++m) {
#pragma unroll
            for (int nn{0}; nn < 2; ++nn) {
#pragma unroll
                for (int j{0}; j < 4; ++j) acc[i][m][nn][j] = 0.0f;
            }
        }
    }
    float db{0.0f};
    const unsigned xa{saddr(xs)};
    const unsigned ga{saddr(gs)};
    const unsigned za{saddr(zs)};
    for (std::uint32_t i{blockIdx.x}; i < n; i += gridDim.x) {
        __syncthreads();
        const bf16* a{act + static_cast<std::size_t>(i) * kNetActPerSample};
        constexpr int kXPer{G::kCin / 8};
        for (int k{tid}; k < G::kInW * G::kInW * kXPer; k += kGradThreads) {
            const int px{k / kXPer};
            const int c{k - px * kXPer};
            *reinterpret_cast<uint4*>(&xs[px * G::kInS + c * 8]) =
                *reinterpret_cast<const uint4*>(a + G::kXOff + px * G::kCin + c * 8);
        }
        for (int k{tid}; k < G::kP * 4; k += kGradThreads) {
            const int px{k >> 2};
            const int c{k & 3};
            *reinterpret_cast<uint4*>(&gs[px * kActS + c * 8]) =
                *reinterpret_cast<const uint4*>(a + G::kGOff + px * kNetC + c * 8);
        }
        __syncthreads();
        if (tid < kNetC) {
            for (int pp{0}; pp < G::kP; ++pp) db = db + __bfloat162float(gs[pp * kActS + tid]);
        }
#pragma unroll 1
        for (int kp{0}; kp < G::kP; kp += 16) {
            unsigned am[2][4];
#pragma unroll
            for (int m{0}; m < 2; ++m) {
                ldsm_x4_t(am[m], ga + 2u * static_cast<unsigned>((kp + (lane & 7) + ((lane >> 4) << 3)) * kActS +
                                                                 m * 16 + ((lane >> 3) & 1) * 8));
            }
#pragma unroll
            for (int pi{0}; pi < kPW; ++pi) {
                const int pair{warp + 8 * pi};
                if (pair < kPairs) {
                    unsigned bb[4];
                    ldsm_x4_t(bb, im2col_row<G::kInW, G::kOutW, G::kStride, G::kPad, G::kCin, G::kInS>(
                                      xa, za, kp + (lane & 7) + ((lane >> 3) & 1) * 8, pair * 16 + (lane >> 4) * 8));
#pragma unroll
                    for (int m{0}; m < 2; ++m) {
                        mma(acc[pi][m][0], am[m], bb[0], bb[1]);
                        mma(acc[pi][m][1], am[m], bb[2], bb[3]);
                    }
                }
            }
        }
    }
    float* out{partial + static_cast<std::size_t>(blockIdx.x) * kNetParams};
#pragma unroll
    for (int pi{0}; pi < kPW; ++pi) {
        const int pair{warp + 8 * pi};
        if (pair >= kPairs) continue;
#pragma unroll
        for (int m{0}; m < 2; ++m) {
#pragma unroll
            for (int nn{0}; nn < 2; ++nn) {
                const int co{m * 16 + (lane >> 2)};
                const int k{pair * 16 + nn * 8 + 2 * (lane & 3)};
                out[G::kWOff + co * G::kK + k] = acc[pi][m][nn][0];
                out[G::kWOff + co * G::kK + k + 1] = acc[pi][m][nn][1];
                out[G::kWOff + (co + 8) * G::kK + k] = acc[pi][m][nn][2];
                out[G::kWOff + (co + 8) * G::kK + k + 1] = acc[pi][m][nn][3];
            }
        }
    }
    if (tid < kNetC) out[kNetBias + (L - 1) * kNetC + tid] = db;
}

struct AdamArgs {
    float* theta;
    float* m;
    float* v;
    std::uint16_t* wbf;
    float lr_t;     // learning rate with both bias corrections folded in
    float eps_t;    // epsilon scaled by the second-moment correction
    int update;
};

// Sums the per-split partial gradients in split order; optionally one Adam
// update of the FP32 master weights and their BF16 copy.
__global__ void acsnet_reduce_kernel(const float* partial, int nsplit, float* grad, AdamArgs a) {
    const int i{static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x)};
    if (i >= kNetParams) return;
    float g{0.0f};
    for (int sp{0}; sp < nsplit; ++sp) g = g + partial[static_cast<std::size_t>(sp) * kNetParams + i];
    if (grad != nullptr) grad[i] = g;
    if (!a.update) return;
    const float m{0.9f * a.m[i] + 0.1f * g};
    const float v{0.999f * a.v[i] + 0.001f * (g * g)};
    a.m[i] = m;
    a.v[i] = v;
    const float t{a.theta[i] - a.lr_t * m / (sqrtf(v) + a.eps_t)};
    a.theta[i] = t;
    if (i < kNetWeights) a.wbf[i] = __bfloat16_as_ushort(__float2bfloat16_rn(t));
}

int sm_count() {
    int dev{0};
    int n{0};
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) !=
                                                   cudaSuccess) {
        return 148;
    }
    return n;
}

}  // namespace

bool acsnet_kernels_init() {
    return cudaFuncSetAttribute(acsnet_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(sizeof(InferSmem))) == cudaSuccess &&
           cudaFuncSetAttribute(acsnet_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(sizeof(TrainSmem))) == cudaSuccess;
}

bool acsnet_infer_launch(const FrontendInputs& in, const NetParamsDev& p, float log2_distance, float margin,
                         const NetDecisionsDev& out, void* stream) {
    const int ntiles{((in.width + 63) >> 6) * ((in.height + 63) >> 6)};
    const int grid{ntiles < sm_count() ? ntiles : sm_count()};
    if (out.tile_order != nullptr &&
        cudaMemsetAsync(out.tile_order + ntiles, 0, 2 * sizeof(std::uint32_t), static_cast<cudaStream_t>(stream)) !=
            cudaSuccess) {
        return false;
    }
    acsnet_infer_kernel<<<grid, kInferThreads, sizeof(InferSmem), static_cast<cudaStream_t>(stream)>>>(
        in, p, log2_distance, margin, out);
    return cudaGetLastError() == cudaSuccess;
}

// Host BF16 rounding (nearest, ties to even), as __float2bfloat16_rn.
std::uint16_t host_bf16(float f) {
    std::uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return 0x7fc0u;
    return static_cast<std::uint16_t>((u + 0x7fffu + ((u >> 16) & 1u)) >> 16);
}

}  // namespace jxb

// ---- SHA-256 (FIPS 180-4), for the weights blob ----
namespace {

class Sha256 {
public:
    void update(const std::uint8_t* d, std::size_t n) {
        for (std::size_t i{0}; i < n; ++i) {
            buf_[fill_++] = d[i];
            if (fill_ == 64) {
                block();
                fill_ = 0;
            }
        }
        len_ += n;
    }

    void finish(std::uint8_t out[32]) {
        const std::uint64_t bits{len_ * 8};
        const std::uint8_t one{0x80};
        update(&one, 1);
        const std::uint8_t z{0};
        while (fill_ != 56) update(&z, 1);
        for (int i{7}; i >= 0; --i) {
            const std::uint8_t b{static_cast<std::uint8_t>(bits >> (8 * i))};
            update(&b, 1);
        }
        for (int i{0}; i < 8; ++i) {
            for (int j{0}; j < 4; ++j) out[4 * i + j] = static_cast<std::uint8_t>(h_[i] >> (24 - 8 * j));
        }
    }

private:
    static std::uint32_t rotr(std::uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

    void block() {
        static constexpr std::uint32_t k[64]{
            0x428a2f98u, 0x71374491u, 0xb5c0fbcfu, 0xe9b5dba5u, 0x3956c25bu, 0x59f111f1u, 0x923f82a4u, 0xab1c5ed5u,
            0xd807aa98u, 0x12835b01u, 0x243185beu, 0x550c7dc3u, 0x72be5d74u, 0x80deb1feu, 0x9bdc06a7u, 0xc19bf174u,
            0xe49b69c1u, 0xefbe4786u, 0x0fc19dc6u, 0x240ca1ccu, 0x2de92c6fu, 0x4a7484aau, 0x5cb0a9dcu, 0x76f988dau,
            0x983e5152u, 0xa831c66du, 0xb00327c8u, 0xbf597fc7u, 0xc6e00bf3u, 0xd5a79147u, 0x06ca6351u, 0x14292967u,
            0x27b70a85u, 0x2e1b2138u, 0x4d2c6dfcu, 0x53380d13u, 0x650a7354u, 0x766a0abbu, 0x81c2c92eu, 0x92722c85u,
            0xa2bfe8a1u, 0xa81a664bu, 0xc24b8b70u, 0xc76c51a3u, 0xd192e819u, 0xd6990624u, 0xf40e3585u, 0x106aa070u,
            0x19a4c116u, 0x1e376c08u, 0x2748774cu, 0x34b0bcb5u, 0x391c0cb3u, 0x4ed8aa4au, 0x5b9cca4fu, 0x682e6ff3u,
            0x748f82eeu, 0x78a5636fu, 0x84c87814u, 0x8cc70208u, 0x90befffau, 0xa4506cebu, 0xbef9a3f7u, 0xc67178f2u};
        std::uint32_t w[64];
        for (int i{0}; i < 16; ++i) {
            w[i] = (static_cast<std::uint32_t>(buf_[4 * i]) << 24) | (static_cast<std::uint32_t>(buf_[4 * i + 1]) << 16) |
                   (static_cast<std::uint32_t>(buf_[4 * i + 2]) << 8) | buf_[4 * i + 3];
        }
        for (int i{16}; i < 64; ++i) {
            const std::uint32_t s0{rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3)};
            const std::uint32_t s1{rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10)};
            w[i] = w[i - 16] + s0 + w[i - 7] + s1;
        }
        std::uint32_t a{h_[0]}, b{h_[1]}, c{h_[2]}, d{h_[3]}, e{h_[4]}, f{h_[5]}, g{h_[6]}, h{h_[7]};
        for (int i{0}; i < 64; ++i) {
            const std::uint32_t s1{rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)};
            const std::uint32_t ch{(e & f) ^ (~e & g)};
            const std::uint32_t t1{h + s1 + ch + k[i] + w[i]};
            const std::uint32_t s0{rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)};
            const std::uint32_t mj{(a & b) ^ (a & c) ^ (b & c)};
            const std::uint32_t t2{s0 + mj};
            h = g;
            g = f;
            f = e;
            e = d + t1;
            d = c;
            c = b;
            b = a;
            a = t1 + t2;
        }
        h_[0] += a;
        h_[1] += b;
        h_[2] += c;
        h_[3] += d;
        h_[4] += e;
        h_[5] += f;
        h_[6] += g;
        h_[7] += h;
    }

    std::uint32_t h_[8]{0x6a09e667u, 0xbb67ae85u, 0x3c6ef372u, 0xa54ff53au,
                        0x510e527fu, 0x9b05688cu, 0x1f83d9abu, 0x5be0cd19u};
    std::uint8_t buf_[64]{};
    std::size_t fill_{0};
    std::uint64_t len_{0};
};

constexpr std::size_t kBlobHeader = 4 + 6 * 4 + 8 * 4;  // magic, six uint32, scale[4], shift[4]
constexpr std::size_t kBlobBytes = kBlobHeader + 4 * static_cast<std::size_t>(jxb::kNetParams) + 32;

std::uint32_t rd32(const std::uint8_t* p) {
    return static_cast<std::uint32_t>(p[0]) | (static_cast<std::uint32_t>(p[1]) << 8) |
           (static_cast<std::uint32_t>(p[2]) << 16) | (static_cast<std::uint32_t>(p[3]) << 24);
}

float rdf(const std::uint8_t* p) {
    const std::uint32_t u{rd32(p)};
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

bool blob_ok(const void* blob, std::size_t size) {
    if (blob == nullptr || size != kBlobBytes) return false;
    const auto* b{static_cast<const std::uint8_t*>(blob)};
    if (std::memcmp(b, "JXBN", 4) != 0 || rd32(b + 4) != 2u || rd32(b + 8) != static_cast<std::uint32_t>(jxb::kNetParams) ||
        rd32(b + 12) != 32u || rd32(b + 16) != 17u || rd32(b + 20) != 80u || rd32(b + 24) != 288u) {
        return false;
    }
    Sha256 h;
    h.update(b, size - 32);
    std::uint8_t d[32];
    h.finish(d);
    if (std::memcmp(d, b + size - 32, 32) != 0) return false;
    for (std::size_t i{28}; i < size - 32; i += 4) {
        if (!std::isfinite(rdf(b + i))) return false;
    }
    return true;
}

class DeviceScope {
public:
    explicit DeviceScope(int device) {
        ok_ = cudaGetDevice(&prev_) == cudaSuccess && cudaSetDevice(device) == cudaSuccess;
    }
    ~DeviceScope() { cudaSetDevice(prev_); }
    bool ok() const { return ok_; }

private:
    int prev_{0};
    bool ok_{false};
};

std::mutex g_init_mutex;
bool g_init[64]{};

bool init_device(int device) {
    if (device < 0 || device >= 64) return false;
    std::lock_guard<std::mutex> lock(g_init_mutex);
    if (!g_init[device]) {
        if (!jxb::acsnet_kernels_init()) return false;
        g_init[device] = true;
    }
    return true;
}

bool valid_device(int device) {
    int n{0};
    return cudaGetDeviceCount(&n) == cudaSuccess && device >= 0 && device < n;
}

}  // namespace

struct cujpegxl_b200_acsnet {
    int device{0};
    void* mem{nullptr};
    jxb::NetParamsDev p{};
};

struct cujpegxl_b200_acsnet_trainer {
    int device{0};
    std::uint32_t max_batch{0};
    int nsplit{0};
    void* mem{nullptr};
    float* theta{nullptr};
    float* m{nullptr};
    float* v{nullptr};
    std::uint16_t* wbf{nullptr};
    float* partial{nullptr};
    __nv_bfloat16* act{nullptr};
    jxb::NetParamsDev p{};
    std::uint32_t steps{0};
};

namespace jxb {

const NetParamsDev* acsnet_params(const cujpegxl_b200_acsnet* net) { return net == nullptr ? nullptr : &net->p; }
int acsnet_device(const cujpegxl_b200_acsnet* net) { return net->device; }

}  // namespace jxb

namespace {

bool batch_dev(const cujpegxl_b200_acsnet_batch* b, std::uint32_t max_batch, bool labels, jxb::NetBatchDev* out) {
    if (b == nullptr || b->n == 0 || b->n > max_batch || b->tiles == nullptr || b->tile_index == nullptr ||
        b->log2_distance == nullptr) {
        return false;
    }
    if (labels && (b->label_class == nullptr || b->label_qf == nullptr)) return false;
    *out = jxb::NetBatchDev{b->tiles, b->tile_index, b->log2_distance, labels ? b->label_class : nullptr,
                            labels ? b->label_qf : nullptr, labels ? b->label_soft : nullptr, b->n};
    return true;
}

int train_grid(std::uint32_t n) {
    const int g{2 * jxb::sm_count()};
    return static_cast<int>(n) < g ? static_cast<int>(n) : g;
}

// Forward + backward-data, the four weight-gradient kernels and the reduction
// (with an Adam update when `lr` > 0).
bool run_gradient(cujpegxl_b200_acsnet_trainer* t, const jxb::NetBatchDev& b, float qf_weight, float* grad,
                  float* stats, float lr, cudaStream_t st) {
    const float inv_batch{1.0f / static_cast<float>(b.n)};
    jxb::acsnet_train_kernel<<<train_grid(b.n), jxb::kNetThreads, sizeof(jxb::TrainSmem), st>>>(
        t->p, b, inv_batch, qf_weight, t->act, nullptr, stats);
    const int ns{static_cast<int>(b.n) < t->nsplit ? static_cast<int>(b.n) : t->nsplit};
    jxb::acsnet_wgrad_kernel<1><<<ns, jxb::kGradThreads, 0, st>>>(t->act, b.n, t->partial);
    jxb::acsnet_wgrad_kernel<2><<<ns, jxb::kGradThreads, 0, st>>>(t->act, b.n, t->partial);
    jxb::acsnet_wgrad_kernel<3><<<ns, jxb::kGradThreads, 0, st>>>(t->act, b.n, t->partial);
    jxb::acsnet_wgrad_kernel<4><<<ns, jxb::kGradThreads, 0, st>>>(t->act, b.n, t->partial);
    jxb::AdamArgs a{t->theta, t->m, t->v, t->wbf, 0.0f, 0.0f, 0};
    if (lr > 0.0f) {
        ++t->steps;
        const double c1{1.0 - std::pow(0.9, static_cast<double>(t->steps))};
        const double c2{1.0 - std::pow(0.999, static_cast<double>(t->steps))};
        // theta -= lr * (m / c1) / (sqrt(v / c2) + 1e-8), rewritten with
        // lr_t = lr * sqrt(c2) / c1 and eps_t = 1e-8 * sqrt(c2).
        a.lr_t = static_cast<float>(lr * std::sqrt(c2) / c1);
        a.eps_t = static_cast<float>(1e-8 * std::sqrt(c2));
        a.update = 1;
    }
    jxb::acsnet_reduce_kernel<<<(jxb::kNetParams + 255) / 256, 256, 0, st>>>(t->partial, ns, grad, a);
    return cudaGetLastError() == cudaSuccess;
}

}  // namespace

extern "C" {

uint32_t cujpegxl_b200_acsnet_param_count(void) { return static_cast<uint32_t>(jxb::kNetParams); }

cujpegxl_status cujpegxl_b200_acsnet_check_blob(const void* blob, size_t size) {
    return blob_ok(blob, size) ? CUJPEGXL_OK : CUJPEGXL_INVALID_ARGUMENT;
}

cujpegxl_status cujpegxl_b200_acsnet_create(const void* blob, size_t size, int32_t device_ordinal,
                                            cujpegxl_b200_acsnet** out_net) {
    if (out_net == nullptr) return CUJPEGXL_INVALID_ARGUMENT;
    *out_net = nullptr;
    if (!blob_ok(blob, size)) return CUJPEGXL_INVALID_ARGUMENT;
    if (!valid_device(device_ordinal)) return CUJPEGXL_NO_DEVICE;
    DeviceScope scope{device_ordinal};
    if (!scope.ok() || !init_device(device_ordinal)) return CUJPEGXL_INTERNAL_ERROR;
    const auto* b{static_cast<const std::uint8_t*>(blob)};
    auto* net{new (std::nothrow) cujpegxl_b200_acsnet};
    if (net == nullptr) return CUJPEGXL_INTERNAL_ERROR;
    net->device = device_ordinal;
    std::vector<std::uint16_t> w(jxb::kNetWeights);
    std::vector<float> bias(4 * jxb::kNetC);
    const std::uint8_t* params{b + kBlobHeader};
    for (int i{0}; i < jxb::kNetWeights; ++i) w[i] = jxb::host_bf16(rdf(params + 4 * i));
    for (int i{0}; i < 4 * jxb::kNetC; ++i) bias[i] = rdf(params + 4 * (jxb::kNetBias + i));
    for (int i{0}; i < 4; ++i) {
        net->p.scale[i] = rdf(b + 28 + 4 * i);
        net->p.shift[i] = rdf(b + 44 + 4 * i);
    }
    const std::size_t wbytes{(w.size() * 2 + 255) & ~static_cast<std::size_t>(255)};
    if (cudaMalloc(&net->mem, wbytes + bias.size() * 4) != cudaSuccess) {
        delete net;
        return CUJPEGXL_INTERNAL_ERROR;
    }
    auto* m{static_cast<std::uint8_t*>(net->mem)};
    if (cudaMemcpy(m, w.data(), w.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(m + wbytes, bias.data(), bias.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(net->mem);
        delete net;
        return CUJPEGXL_INTERNAL_ERROR;
    }
    net->p.w = reinterpret_cast<const std::uint16_t*>(m);
    net->p.bias = reinterpret_cast<const float*>(m + wbytes);
    *out_net = net;
    return CUJPEGXL_OK;
}

void cujpegxl_b200_acsnet_destroy(cujpegxl_b200_acsnet* net) {
    if (net == nullptr) return;
    DeviceScope scope{net->device};
    cudaFree(net->mem);
    delete net;
}

cujpegxl_status cujpegxl_b200_acsnet_trainer_create(const float* params, const float* norm, uint32_t max_batch,
                                                    int32_t device_ordinal,
                                                    cujpegxl_b200_acsnet_trainer** out_trainer) {
    if (out_trainer == nullptr) return CUJPEGXL_INVALID_ARGUMENT;
    *out_trainer = nullptr;
    if (params == nullptr || norm == nullptr || max_batch == 0 || max_batch > (1u << 20)) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    for (int i{0}; i < jxb::kNetParams; ++i) {
        if (!std::isfinite(params[i])) return CUJPEGXL_INVALID_ARGUMENT;
    }
    if (!valid_device(device_ordinal)) return CUJPEGXL_NO_DEVICE;
    DeviceScope scope{device_ordinal};
    if (!scope.ok() || !init_device(device_ordinal)) return CUJPEGXL_INTERNAL_ERROR;
    auto* t{new (std::nothrow) cujpegxl_b200_acsnet_trainer};
    if (t == nullptr) return CUJPEGXL_INTERNAL_ERROR;
    t->device = device_ordinal;
    t->max_batch = max_batch;
    t->nsplit = 2 * jxb::sm_count();
    auto a256 = [](std::size_t v) { return (v + 255) & ~static_cast<std::size_t>(255); };
    const std::size_t np{static_cast<std::size_t>(jxb::kNetParams)};
    const std::size_t o_theta{0};
    const std::size_t o_m{o_theta + a256(np * 4)};
    const std::size_t o_v{o_m + a256(np * 4)};
    const std::size_t o_w{o_v + a256(np * 4)};
    const std::size_t o_part{o_w + a256(np * 2)};
    const std::size_t o_act{o_part + a256(np * 4 * static_cast<std::size_t>(t->nsplit))};
    const std::size_t total{o_act + a256(static_cast<std::size_t>(max_batch) * jxb::kNetActPerSample * 2)};
    if (cudaMalloc(&t->mem, total) != cudaSuccess) {
        delete t;
        return CUJPEGXL_INTERNAL_ERROR;
    }
    auto* m{static_cast<std::uint8_t*>(t->mem)};
    t->theta = reinterpret_cast<float*>(m + o_theta);
    t->m = reinterpret_cast<float*>(m + o_m);
    t->v = reinterpret_cast<float*>(m + o_v);
    t->wbf = reinterpret_cast<std::uint16_t*>(m + o_w);
    t->partial = reinterpret_cast<float*>(m + o_part);
    t->act = reinterpret_cast<__nv_bfloat16*>(m + o_act);
    std::vector<std::uint16_t> w(jxb::kNetWeights);
    for (int i{0}; i < jxb::kNetWeights; ++i) w[i] = jxb::host_bf16(params[i]);
    if (cudaMemcpy(t->theta, params, np * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(t->m, 0, np * 4) != cudaSuccess || cudaMemset(t->v, 0, np * 4) != cudaSuccess ||
        cudaMemcpy(t->wbf, w.data(), w.size() * 2, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(t->mem);
        delete t;
        return CUJPEGXL_INTERNAL_ERROR;
    }
    t->p.w = t->wbf;
    t->p.bias = t->theta + jxb::kNetBias;
    for (int i{0}; i < 4; ++i) {
        t->p.scale[i] = norm[i];
        t->p.shift[i] = norm[4 + i];
    }
    *out_trainer = t;
    return CUJPEGXL_OK;
}

void cujpegxl_b200_acsnet_trainer_destroy(cujpegxl_b200_acsnet_trainer* trainer) {
    if (trainer == nullptr) return;
    DeviceScope scope{trainer->device};
    cudaFree(trainer->mem);
    delete trainer;
}

cujpegxl_status cujpegxl_b200_acsnet_trainer_forward(cujpegxl_b200_acsnet_trainer* trainer,
                                                     const cujpegxl_b200_acsnet_batch* batch, float* out,
                                                     uintptr_t stream) {
    jxb::NetBatchDev b{};
    if (trainer == nullptr || out == nullptr || !batch_dev(batch, trainer->max_batch, false, &b)) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    DeviceScope scope{trainer->device};
    if (!scope.ok()) return CUJPEGXL_INTERNAL_ERROR;
    jxb::acsnet_train_kernel<<<train_grid(b.n), jxb::kNetThreads, sizeof(jxb::TrainSmem),
                               reinterpret_cast<cudaStream_t>(stream)>>>(trainer->p, b, 0.0f, 0.0f, trainer->act, out,
                                                                         nullptr);
    return cudaGetLastError() == cudaSuccess ? CUJPEGXL_OK : CUJPEGXL_INTERNAL_ERROR;
}

cujpegxl_status cujpegxl_b200_acsnet_trainer_gradient(cujpegxl_b200_acsnet_trainer* trainer,
                                                      const cujpegxl_b200_acsnet_batch* batch, float qf_weight,
                                                      float* grad, float* stats, uintptr_t stream) {
    jxb::NetBatchDev b{};
    if (trainer == nullptr || grad == nullptr || !(qf_weight >= 0.0f) ||
        !batch_dev(batch, trainer->max_batch, true, &b)) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    DeviceScope scope{trainer->device};
    if (!scope.ok()) return CUJPEGXL_INTERNAL_ERROR;
    return run_gradient(trainer, b, qf_weight, grad, stats, 0.0f, reinterpret_cast<cudaStream_t>(stream))
               ? CUJPEGXL_OK
               : CUJPEGXL_INTERNAL_ERROR;
}

cujpegxl_status cujpegxl_b200_acsnet_trainer_step(cujpegxl_b200_acsnet_trainer* trainer,
                                                  const cujpegxl_b200_acsnet_batch* batch, float qf_weight,
                                                  float learning_rate, float* stats, uintptr_t stream) {
    jxb::NetBatchDev b{};
    if (trainer == nullptr || !(qf_weight >= 0.0f) || !(learning_rate > 0.0f) ||
        !batch_dev(batch, trainer->max_batch, true, &b)) {
        return CUJPEGXL_INVALID_ARGUMENT;
    }
    DeviceScope scope{trainer->device};
    if (!scope.ok()) return CUJPEGXL_INTERNAL_ERROR;
    return run_gradient(trainer, b, qf_weight, nullptr, stats, learning_rate, reinterpret_cast<cudaStream_t>(stream))
               ? CUJPEGXL_OK
               : CUJPEGXL_INTERNAL_ERROR;
}

cujpegxl_status cujpegxl_b200_acsnet_trainer_params(cujpegxl_b200_acsnet_trainer* trainer, float* params) {
    if (trainer == nullptr || params == nullptr) return CUJPEGXL_INVALID_ARGUMENT;
    DeviceScope scope{trainer->device};
    if (!scope.ok() || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(params, trainer->theta, static_cast<std::size_t>(jxb::kNetParams) * 4, cudaMemcpyDeviceToHost) !=
            cudaSuccess) {
        return CUJPEGXL_INTERNAL_ERROR;
    }
    return CUJPEGXL_OK;
}

}  // extern "C"
