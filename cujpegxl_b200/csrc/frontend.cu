// Fused frontend kernel (one CTA per 64x64 colour tile) and its host setup.
//
// Arithmetic contract. This file is compiled with -fmad=false: a*b+c is two
// rounded operations unless written as jx_fma. Every float expression below is
// the canonical definition that the CPU restatement in oracle/ reproduces
// operation for operation, so the kernel's integer outputs (quant field,
// transform choice, CfL maps, quantised coefficients) match it bit for bit.
// Where the reference has a host twin of a stage (transform selection,
// src/transform_select_impl.cuh; LLF -> DC, src/vardct_layout.h) the twin's
// exact arithmetic is used, including its lack of FMA and its partial-sum
// order, so results equal the twin's too.

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "frontend.cuh"
#include "jxl_constants.cuh"
#include "jxl_math.cuh"
#include "f16_mixed.cuh"
#include "ratio_div.cuh"
#include "xyb.cuh"

namespace jxb {
namespace {

#include "jxl_dequant_tables.inc"

constexpr int kThreads = 256;
constexpr int kTile = 64;
constexpr int kHalo = 2;
constexpr int kXs = kTile + 2 * kHalo;  // 68: stride of the unsharpened XYB tile
constexpr int kXplane = kXs * kXs;
// 68: stride of the sharpened tile, a multiple of 4 floats so that every
// block row starts 16-byte aligned for the DCT passes' vector loads.
constexpr int kSs = kTile + 4;
constexpr int kSplane = kTile * kSs;
constexpr int kRegionAFloats = 3 * kXplane;  // 13872
// FP16 coefficients of the tile: 64 covered-block slots per block, padded to
// 66 so that lanes walking different blocks at the same slot hit different
// shared-memory banks. Channel c's plane lies over sharpened plane c (region
// B), kCoefStride halves apart.
constexpr int kCoefBlock = 66;
constexpr int kCoefPlane = 64 * kCoefBlock;
constexpr int kCoefStride = 2 * kSplane;
static_assert(kCoefPlane <= kCoefStride, "a coefficient plane exceeds its sharpened plane");
// Final-DCT row scratch of one channel (floats); the three channels' lie
// side by side in region A.
constexpr int kDrowsChannel = 64 * 72;
static_assert(3 * kDrowsChannel <= kRegionAFloats, "final-DCT scratch exceeds region A");
// Row stride of one first block's row-pass output in the final-DCT scratch:
// 36 for DCT32 (16-byte aligned rows for the column pass's vector loads; one
// block per warp, so lanes stay on distinct banks), N + 1 for DCT16 and DCT8,
// whose warps span several blocks. Each 32x32 region then needs at most
// 32 * 36 = 16 * 8 * 9 floats, so the scratch bound above still holds.
template <int N>
constexpr int kDrowsStride = N == 32 ? 36 : N + 1;

// Selection bases: double-precision DCT-II basis narrowed to float
// (basis[k*n + t], src/transform_select.cu:29-37). Final-DCT bases: the float
// basis of src/frontend_transform.cu:104-106 (cosf of a float argument).
// Stored as pairs of consecutive frequencies, {basis[k][t], basis[k+1][t]} at
// (k/2)*n + t for even k, so that the DCT passes compute two coefficients per
// packed f32x2 instruction (per component the same rounding as the scalar
// instruction, so the results are those of the scalar chains).
__constant__ float2 c_sel8[32];
__constant__ float2 c_sel16[128];
__constant__ float2 c_sel32[512];
__constant__ float2 c_dct8[32];
__constant__ float2 c_dct16[128];
__constant__ float2 c_dct32[512];

template <int N, bool kSel>
__device__ __forceinline__ float2 basis2(int i) {
    if (kSel) {
        return N == 8 ? c_sel8[i] : (N == 16 ? c_sel16[i] : c_sel32[i]);
    }
    return N == 8 ? c_dct8[i] : (N == 16 ? c_dct16[i] : c_dct32[i]);
}

__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }

// Rate-proxy table entries kept in shared memory: quantised magnitudes below
// this are by far the most frequent.
constexpr int kLog2Cached = 256;

struct Small {
    float pre[256];       // AQ pre-erosion cells, 16x16 over the tile
    float log2_small[kLog2Cached];  // log2f(1 + i), the first entries of the rate table
    float cost8[64];
    float cost16[16];
    float cost32[4];
    float cfl[3][64];
    float aq_sums[4][64];  // per block: HF sum, gamma sum, blue sum, eroded mask
    int qf[64];
    int nz[3][64];
    int fb_off[64];       // final-DCT scratch offset of each listed first-block
    unsigned char fb_list[64];
    unsigned char owner[64];
    signed char acs[64];
    int n32, n16, n8;
    signed char net[4];   // learned split class of each 32x32 region, -1 = RD heuristic
    float2 pow_lut[6];    // factor table of jx_pow24_2, for the packed sRGB transfer
};

// Region (0..3, raster) of the tile that holds tile block lb.
__device__ __forceinline__ int region_of_block(int lb) { return ((lb >> 5) << 1) | ((lb & 7) >> 2); }

constexpr std::size_t kSmemBytes =
    sizeof(float) * (kRegionAFloats + 3 * kSplane) + sizeof(Small);
// The batch kernel's single-tile CTAs run two per SM: 228 KB of shared
// memory, 1 KB of it reserved per CTA.
static_assert(2 * (kSmemBytes + 1024) <= 228 * 1024, "two frontend CTAs no longer fit on one SM");
// One tile's shared memory, rounded to 16 bytes: the single-frame kernel runs
// two tiles per CTA, one per half of its threads, at this stride.
constexpr std::size_t kTileSmemStride = (kSmemBytes + 15) / 16 * 16;
// The single-frame kernel's CTA: two tiles of kThreads threads each, all of
// an SM's shared memory (227 KB per CTA at most).
constexpr int kPairThreads = 2 * kThreads;
static_assert(2 * kTileSmemStride <= 227 * 1024, "two tiles no longer fit in one CTA");

// Synchronises the kThreads threads of one tile on named barrier `bar` (1 or
// 2; barrier 0 is __syncthreads), with the ordering of shared memory that
// __syncthreads gives.
__device__ __forceinline__ void tile_sync(int bar) {
    asm volatile("bar.sync %0, %1;" ::"r"(bar), "n"(kThreads) : "memory");
}

// Chroma window of a tile in shared memory: kChromaWin x kChromaWin (cb, cr)
// pairs starting kChromaMargin chroma samples before the tile's first.
constexpr int kChromaMargin = 2;
constexpr int kChromaWin = kTile / 2 + 2 * kChromaMargin;  // 36

// a / w for a weight w of the dequantisation tables, from w_inv = RN(1 / w)
// by Markstein's method: q0 = RN(a * w_inv), the residual a - q0 * w is exact
// in one FMA, and RN(q0 + residual * w_inv) is the IEEE quotient RN(a / w).
// That equality is checked for every weight of the tables (all three sizes
// and channels) and every significand of a by
// tests/cpu_checks/quant_div_check.c; both sides scale exactly with a's
// exponent and are odd in a, so it holds for every a whose quotient and
// residual stay normal, which includes every |a| > w / 2 the quantiser
// divides. (The selection's quantiser keeps the IEEE division: its quotients
// are formed in an out-of-line function, where loading the reciprocal cost
// more than the division.)
__device__ __forceinline__ float div_weight(float a, float w, float w_inv) {
    const float q0{a * w_inv};
    return jx_fma(jx_fma(-q0, w, a), w_inv, q0);
}

// lrintf((v * qgsf) / w) for a positive weight w (src/frontend_quantize.cu:
// 165-178), with no branch: the quotient is exact wherever it can round away
// from zero (|v * qgsf| >= w / 2 keeps div_weight's intermediates normal), and
// where the dividend is so small that they are not, the quotient is far below
// 1/2 and rounds to zero either way. (Without the zero fast path the lanes of
// a warp no longer diverge: 3% fewer cycles in the phase.)
__device__ __forceinline__ int quantize(float v, float qgsf, float w, float w_inv) {
    return static_cast<int>(lrintf(div_weight(v * qgsf, w, w_inv)));
}

// RatioOfDerivativesOfCubicRootToSimpleGamma (src/adaptive_quant_impl.cuh:44-55).
template <bool kInvert>
__device__ __forceinline__ float ratio_gamma(float v) {
    v = v < 0.0f ? 0.0f : v;
    const float v2{v * v};
    const float num{jx_fma(kRatioNumMul, v2, kRatioEps)};
    const float den{jx_fma(kRatioDenMul * v, v2, kRatioVOffset)};
    return kInvert ? num / den : den / num;
}

// src/adaptive_quant_impl.cuh:63-76.
__device__ __forceinline__ float compute_mask(float out_val) {
    const float v1{fmaxf(out_val * kMaskMul0, 1e-3f)};
    const float v2{1.0f / (v1 + kMaskOffset2)};
    const float v3{1.0f / jx_fma(v1, v1, kMaskOffset3)};
    const float v4{1.0f / jx_fma(v1, v1, kMaskOffset4)};
    float r{jx_fma(kMaskMul4, v4, kMaskBase)};
    r = jx_fma(kMaskMul2, v2, r);
    r = jx_fma(kMaskMul3, v3, r);
    return r;
}

__device__ __forceinline__ void swap_if(float& a, float& b) {
    if (a > b) {
        const float t{a};
        a = b;
        b = t;
    }
}

__device__ __forceinline__ void keep_min4(float v, float& m0, float& m1, float& m2, float& m3) {
    if (v < m3) {
        if (v < m0) {
            m3 = m2; m2 = m1; m1 = m0; m0 = v;
        } else if (v < m1) {
            m3 = m2; m2 = m1; m1 = v;
        } else if (v < m2) {
            m3 = m2; m2 = v;
        } else {
            m3 = v;
        }
    }
}

// FuzzyErosion of cell (cx, cy) of one 32x32 AQ tile whose 8x8 cells start at
// (sx0, sy0) in the 16x16 tile grid: weighted four smallest of the 3x3
// neighbourhood clamped to the AQ tile (src/frontend_fused.cu:35-53).
__device__ float erosion_cell(const float* pre, int sx0, int sy0, int cx, int cy, float km0,
                              float km1, float km2, float km3) {
    const int xm{cx > 0 ? cx - 1 : cx};
    const int xp{cx + 1 < 8 ? cx + 1 : cx};
    const int ym{cy > 0 ? cy - 1 : cy};
    const int yp{cy + 1 < 8 ? cy + 1 : cy};
    auto at = [&](int x, int y) { return pre[(sy0 + y) * 16 + sx0 + x]; };
    float m0{at(cx, cy)};
    float m1{at(xm, cy)};
    float m2{at(xp, cy)};
    float m3{at(xm, ym)};
    swap_if(m0, m1);
    swap_if(m0, m2);
    swap_if(m0, m3);
    swap_if(m1, m2);
    swap_if(m1, m3);
    swap_if(m2, m3);
    keep_min4(at(cx, ym), m0, m1, m2, m3);
    keep_min4(at(xp, ym), m0, m1, m2, m3);
    keep_min4(at(xm, yp), m0, m1, m2, m3);
    keep_min4(at(cx, yp), m0, m1, m2, m3);
    keep_min4(at(xp, yp), m0, m1, m2, m3);
    float r{km0 * m0};
    r = jx_fma(km1, m1, r);
    r = jx_fma(km2, m2, r);
    r = jx_fma(km3, m3, r);
    return r;
}

// warp_tree on both components at once (two shuffles, one packed add per
// step); each component's sum is warp_tree's.
__device__ __forceinline__ float2 warp_tree2(float2 v) {
#pragma unroll
    for (int off{16}; off > 0; off >>= 1) {
        v = __fadd2_rn(v, make_float2(__shfl_down_sync(0xffffffffu, v.x, off), __shfl_down_sync(0xffffffffu, v.y, off)));
    }
    return v;
}

// ratio_gamma<true> on both components.
__device__ __forceinline__ float2 ratio_gamma_inv2(float2 v) {
    v = make_float2(v.x < 0.0f ? 0.0f : v.x, v.y < 0.0f ? 0.0f : v.y);
    const float2 v2{__fmul2_rn(v, v)};
    const float2 num{__ffma2_rn(f2dup(kRatioNumMul), v2, f2dup(kRatioEps))};
    const float2 den{__ffma2_rn(__fmul2_rn(f2dup(kRatioDenMul), v), v2, f2dup(kRatioVOffset))};
    return div2_ratio(num, den);
}

// Sum over the 32 lanes with the shfl_down pairing (offsets 16..1); the total
// lands in lane 0.
__device__ __forceinline__ float warp_tree(float v) {
#pragma unroll
    for (int off{16}; off > 0; off >>= 1) {
        v = v + __shfl_down_sync(0xffffffffu, v, off);
    }
    return v;
}

// Row pass of an N-point separable DCT: dst[fx*(N+1)] for fx in [F0, F1) from
// one pixel row. Selection bases accumulate without FMA (the host twin's
// arithmetic); final-DCT bases accumulate with FMA. Coefficients fx and fx+1
// share each packed instruction; each is its own chain in c order.
// src is 16-byte aligned (block rows of the sharpened planes are). The
// outputs of frequency fx go to dst[fx * stride]: stride N + 1 for the
// selection scratch, kDrowsStride<N> for the final DCT.
template <int N, int F0, int F1, bool kSel>
__device__ __forceinline__ void row_pass(const float* src, float* dst) {
    static_assert(F0 % 2 == 0 && F1 % 2 == 0, "pairs of frequencies");
    constexpr int kStride{kSel ? N + 1 : kDrowsStride<N>};
    float2 p[N];
#pragma unroll
    for (int c{0}; c < N; c += 4) {
        const float4 v{*reinterpret_cast<const float4*>(src + c)};
        p[c] = dup2(v.x);
        p[c + 1] = dup2(v.y);
        p[c + 2] = dup2(v.z);
        p[c + 3] = dup2(v.w);
    }
#pragma unroll
    for (int fx{F0}; fx < F1; fx += 2) {
        float2 s{0.0f, 0.0f};
#pragma unroll
        for (int c{0}; c < N; ++c) {
            if (kSel) {
                s = __fadd2_rn(s, __fmul2_rn(basis2<N, true>((fx >> 1) * N + c), p[c]));
            } else {
                s = __ffma2_rn(basis2<N, false>((fx >> 1) * N + c), p[c], s);
            }
        }
        dst[fx * kStride] = s.x;
        dst[(fx + 1) * kStride] = s.y;
    }
}

// Column pass of the selection proxy fused with its quantiser: for fy in
// [Y0, Y1) computes coefficient (fx, fy), quantises it with the DCT8 Y weight
// sampled at the coefficient's frequency and stores its distortion and rate
// contributions (zero for the low-frequency corner), as in block_ac_cost
// (src/transform_select_impl.cuh:80-106).
// Distortion and rate of a selection coefficient whose quantum may be non-zero
// (block_ac_cost, src/transform_select_impl.cuh:80-106). Kept out of line:
// the unrolled column passes call it from hundreds of sites, and one shared
// body keeps their code small enough for the instruction caches.
__device__ __noinline__ float2 sel_cost_nonzero(float coeff, float scaled, float w, float qgsf, const float* l2t,
                                                const float* l2s) {
    const float q{rintf(scaled / w)};
    const float err{(q * w) / qgsf - coeff};
    float rt{0.0f};
    if (q != 0.0f) {
        int a{static_cast<int>(fabsf(q))};
        a = a < kLog2TableSize ? a : kLog2TableSize - 1;
        rt = 1.0f + (a < kLog2Cached ? l2s[a] : l2t[a]);
    }
    return make_float2(err * err, rt);
}

template <int N, int Y0, int Y1>
__device__ __forceinline__ void sel_col(const float* rows_fx, float* cd_fx, float* cr_fx, int fx,
                                        float qgsf, const float* wsel, const float* l2t,
                                        const float* l2s) {
    static_assert(Y0 % 2 == 0 && Y1 % 2 == 0, "pairs of frequencies");
    float2 rr[N];
#pragma unroll
    for (int r{0}; r < N; ++r) {
        rr[r] = dup2(rows_fx[r]);
    }
#pragma unroll
    for (int fy0{Y0}; fy0 < Y1; fy0 += 2) {
        float2 c2{0.0f, 0.0f};
#pragma unroll
        for (int r{0}; r < N; ++r) {
            c2 = __fadd2_rn(c2, __fmul2_rn(basis2<N, true>((fy0 >> 1) * N + r), rr[r]));
        }
        // Weights, scaled values, half-weights and squares of the pair at once
        // (fx * N + fy0 is even: one 8-byte weight load).
        const float2 w2{*reinterpret_cast<const float2*>(wsel + fx * N + fy0)};
        const float2 sc2{__fmul2_rn(c2, f2dup(qgsf))};
        const float2 hw2{__fmul2_rn(f2dup(0.5f), w2)};
        const float2 sq2{__fmul2_rn(c2, c2)};
#pragma unroll
        for (int h{0}; h < 2; ++h) {
            const int fy{fy0 + h};
            const float coeff{h == 0 ? c2.x : c2.y};
            float d{0.0f};
            float rt{0.0f};
            if (!(fx < N / 8 && fy < N / 8)) {
                const float w{h == 0 ? w2.x : w2.y};
                const float scaled{h == 0 ? sc2.x : sc2.y};
                if (fabsf(scaled) <= (h == 0 ? hw2.x : hw2.y)) {
                    // |scaled / w| <= 1/2 rounds to a quotient of at most 1/2,
                    // so q is zero and err is -coeff exactly: the same d, no
                    // rate.
                    d = h == 0 ? sq2.x : sq2.y;
                } else {
                    const float2 dr{sel_cost_nonzero(coeff, scaled, w, qgsf, l2t, l2s)};
                    d = dr.x;
                    rt = dr.y;
                }
            }
            cd_fx[fy] = d;
            cr_fx[fy] = rt;
        }
    }
}

// Final-DCT column pass: coefficients (fx, fy) for fy in [Y0, Y1), rounded to
// FP16 and stored at their covered-block slot in the tile's coefficient
// buffer (src/frontend_transform.cu:252-262).
template <int N, int Y0, int Y1>
__device__ __forceinline__ void dct_col(const float* rows_fx, __half* coef, int fx, int fbx,
                                        int fby) {
    static_assert(Y0 % 2 == 0 && Y1 % 2 == 0, "pairs of frequencies");
    float2 rr[N];
    if constexpr (kDrowsStride<N> % 4 == 0) {
        // 16-byte aligned rows: four samples per load.
#pragma unroll
        for (int r{0}; r < N; r += 4) {
            const float4 v{*reinterpret_cast<const float4*>(rows_fx + r)};
            rr[r] = dup2(v.x);
            rr[r + 1] = dup2(v.y);
            rr[r + 2] = dup2(v.z);
            rr[r + 3] = dup2(v.w);
        }
    } else {
#pragma unroll
        for (int r{0}; r < N; ++r) {
            rr[r] = dup2(rows_fx[r]);
        }
    }
    constexpr int side{N / 8};
#pragma unroll
    for (int fy{Y0}; fy < Y1; fy += 2) {
        float2 c2{0.0f, 0.0f};
#pragma unroll
        for (int r{0}; r < N; ++r) {
            c2 = __ffma2_rn(basis2<N, false>((fy >> 1) * N + r), rr[r], c2);
        }
        // raw and raw + 1 share their 64-slot group (raw is even), and the
        // pair's slot is 4-byte aligned (kCoefBlock is even).
        const int raw{fx * N + fy};
        const int q{raw >> 6};
        const int lb{(fby + q / side) * 8 + fbx + q % side};
        *reinterpret_cast<__half2*>(coef + lb * kCoefBlock + (raw & 63)) = __floats2half2_rn(c2.x, c2.y);
    }
}

// One CfL sum of a side-N first block lb over its non-LLF coefficients
// (src/frontend_quantize.cu:49-74 sums them in raw order in one chain), here
// across a warp: lane l accumulates raw positions l, l + 32, l + 64, ... in
// that order, then the 32 partial sums meet in an xor-butterfly tree (the same
// total on every lane). kWhich 0 sums x*y, 1 sums y*y and 2 sums (b - y)*y,
// each product an FMA of the widened FP16 operands into the lane's partial. An
// LLF position contributes fma(0, y, acc): it adds an exact zero.
template <int N, int kWhich>
__device__ __forceinline__ float cfl_sum_warp(const __half* coef, int lb, int lane) {
    constexpr int kSide{N / 8};
    float acc{0.0f};
#pragma unroll
    for (int k{0}; k < N * N / 32; ++k) {
        const int raw{lane + 32 * k};
        const int q{raw >> 6};
        const int l{lb + (q / kSide) * 8 + q % kSide};
        const int at{l * kCoefBlock + (raw & 63)};
        const bool llf{(raw / N) < kSide && (raw % N) < kSide};
        const auto yh{__half_as_ushort(coef[kCoefStride + at])};
        if (kWhich == 2) {
            const float yr{__half2float(__ushort_as_half(yh))};
            float a{add_f16(__half_as_ushort(coef[2 * kCoefStride + at]), -yr)};
            a = llf ? 0.0f : a;
            acc = jx_fma(a, yr, acc);
        } else {
            auto ah{kWhich == 0 ? __half_as_ushort(coef[at]) : yh};
            ah = llf ? static_cast<unsigned short>(0) : ah;
            acc = fma_f16(ah, yh, acc);
        }
    }
#pragma unroll
    for (int off{16}; off > 0; off >>= 1) acc = acc + __shfl_xor_sync(0xffffffffu, acc, off);
    return acc;
}

template <int N>
__device__ __forceinline__ float cfl_sum_kind(const __half* coef, int lb, int which, int lane) {
    return which == 0 ? cfl_sum_warp<N, 0>(coef, lb, lane)
                      : (which == 1 ? cfl_sum_warp<N, 1>(coef, lb, lane) : cfl_sum_warp<N, 2>(coef, lb, lane));
}

// DC of the 8x8 position (ox, oy) of a first block f of side 8M from its
// MxM low-frequency corner, per channel, in double as the host twin computes
// it (src/vardct_layout.h:88-111): the sum over fx, then fy, of
// (((ob[fx][ox] * ob[fy][oy]) * c) * s[fx]) * s[fy], times M. The basis
// product does not depend on the channel, so it is formed once for all three
// (the same rounded value each channel would form).
template <int M>
__device__ __forceinline__ void llf_to_dc(const __half* coef, int f, int ox, int oy, const double* ob,
                                          float dcv[3]) {
    constexpr int kN{8 * M};
    constexpr double kS16[2]{1.0, 0.901764195028874394};
    constexpr double kS32[4]{1.0, 0.974886821136879522, 0.901764195028874394, 0.787054918159101335};
    double bx[M];
    double by[M];
#pragma unroll
    for (int i{0}; i < M; ++i) {
        bx[i] = ob[i * 4 + ox];
        by[i] = ob[i * 4 + oy];
    }
    double ab[M][M];
#pragma unroll
    for (int fx{0}; fx < M; ++fx) {
#pragma unroll
        for (int fy{0}; fy < M; ++fy) ab[fx][fy] = bx[fx] * by[fy];
    }
#pragma unroll
    for (int c{0}; c < 3; ++c) {
        double sum{0.0};
#pragma unroll
        for (int fx{0}; fx < M; ++fx) {
#pragma unroll
            for (int fy{0}; fy < M; ++fy) {
                const int raw{fx * kN + fy};
                const int q{raw >> 6};
                const int blk{f + (q >> (M >> 1)) * 8 + (q & (M - 1))};
                const double cv{__half2float(coef[c * kCoefStride + blk * kCoefBlock + (raw & 63)])};
                const double sx{M == 2 ? kS16[fx] : kS32[fx]};
                const double sy{M == 2 ? kS16[fy] : kS32[fy]};
                sum = sum + ((ab[fx][fy] * cv) * sx) * sy;
            }
        }
        dcv[c] = static_cast<float>(static_cast<double>(M) * sum);
    }
}

// The whole frontend of the 64x64 tile (tx, ty) of one frame; `smem` is the
// CTA's dynamic shared memory (kSmemBytes). The caller synchronises before
// the CTA starts another tile.
__device__ __forceinline__ void frontend_tile(const FrontendInputs& in, const FrontendScalars& sc,
                                              const FrontendTables& tb, const FrontendOutputs& out, int tx,
                                              int ty, float* smem, int bar) {
    // Region A: the XYB planes, later the selection and final-DCT row
    // scratch. Region B: the sharpened planes, later the FP16 coefficients
    // and the NV12 window before both.
    float* xyb{smem};                                // [3][68*68]
    float* shp{smem + kRegionAFloats};               // [3][64*kSs]
    Small& sm{*reinterpret_cast<Small*>(smem + kRegionAFloats + 3 * kSplane)};

    const int tid{static_cast<int>(threadIdx.x) & (kThreads - 1)};
    const int lane{tid & 31};
    const int warp{tid >> 5};
    const int W{in.width};
    const int H{in.height};
    const int bw{W >> 3};
    const int bh{H >> 3};
    const int nblocks{bw * bh};
    const int px0{tx * kTile};
    const int py0{ty * kTile};
    const int bx0{tx * 8};
    const int by0{ty * 8};

    // ---- 1. NV12 -> XYB over the tile and a 2-pixel halo (clamped coordinates).
    // 1a. Stage the NV12 window in region B, which is free until gaborish: the
    // luma of every halo pixel and the chroma pairs of chroma columns and rows
    // cx0..cx0+35 and cy0..cy0+35, each at its clamped coordinate. All loads
    // are independent, so their latencies overlap.
    std::uint8_t* win_luma{reinterpret_cast<std::uint8_t*>(shp)};
    std::uint8_t* win_chroma{win_luma + kXplane};
    const int cx0{(px0 >> 1) - kChromaMargin};
    const int cy0{(py0 >> 1) - kChromaMargin};
    {
        const int cw{W >> 1};
        const int ch{H >> 1};
        // The rate-table entry and the learned class are loaded here and
        // stored after the window, so that their latency overlaps the
        // window's.
        static_assert(kLog2Cached == kThreads, "one cached rate-table entry per thread");
        const float log2_entry{tb.log2_1p[tid]};
        signed char net_entry{-1};
        if (tid < 4) {
            const int rw{(bw + 3) >> 2};
            const int rx{2 * tx + (tid & 1)};
            const int ry{2 * ty + (tid >> 1)};
            if (in.net_class != nullptr && rx < rw && ry < ((bh + 3) >> 2)) net_entry = in.net_class[ry * rw + rx];
        }
        // Interior tiles whose window needs no clamping, with 4-byte aligned
        // rows, load whole 32-bit words: luma bytes px0-4 .. px0+67 of each
        // row (the window starts 2 bytes in), chroma pairs cx0 .. cx0+35
        // (bytes px0-4 .. px0+67, word aligned).
        const bool aligned{((reinterpret_cast<std::uintptr_t>(in.luma) | in.luma_pitch |
                             reinterpret_cast<std::uintptr_t>(in.chroma) | in.chroma_pitch) & 3u) == 0};
        // Each thread issues all of its loads before its first shared-memory
        // store, so that it waits for one memory latency rather than one per
        // loop iteration.
        if (aligned && px0 >= 4 && py0 >= 4 && px0 + 68 <= W && py0 + 68 <= H) {
            constexpr int kLumaWords{kXs / 4};        // 17 output words per luma row
            constexpr int kChromaWords{kChromaWin / 2};  // 18 words per chroma row
            constexpr int kLumaItems{kXs * kLumaWords};
            constexpr int kChromaItems{kChromaWin * kChromaWords};
            constexpr int kLumaPer{(kLumaItems + kThreads - 1) / kThreads};
            constexpr int kChromaPer{(kChromaItems + kThreads - 1) / kThreads};
            std::uint32_t lo[kLumaPer], hi[kLumaPer], cv[kChromaPer];
#pragma unroll
            for (int j{0}; j < kLumaPer; ++j) {
                const int i{tid + j * kThreads};
                if (i < kLumaItems) {
                    const int row{i / kLumaWords};
                    const int w{i - row * kLumaWords};
                    const auto* src{reinterpret_cast<const std::uint32_t*>(
                        in.luma + static_cast<std::size_t>(py0 - kHalo + row) * in.luma_pitch + px0 - 4)};
                    lo[j] = __ldg(&src[w]);
                    hi[j] = __ldg(&src[w + 1]);
                }
            }
#pragma unroll
            for (int j{0}; j < kChromaPer; ++j) {
                const int i{tid + j * kThreads};
                if (i < kChromaItems) {
                    const int row{i / kChromaWords};
                    const int w{i - row * kChromaWords};
                    const auto* src{reinterpret_cast<const std::uint32_t*>(
                        in.chroma + static_cast<std::size_t>(cy0 + row) * in.chroma_pitch + 2 * cx0)};
                    cv[j] = __ldg(&src[w]);
                }
            }
            auto* lw{reinterpret_cast<std::uint32_t*>(win_luma)};  // word i = row * kLumaWords + w
#pragma unroll
            for (int j{0}; j < kLumaPer; ++j) {
                const int i{tid + j * kThreads};
                if (i < kLumaItems) lw[i] = __funnelshift_r(lo[j], hi[j], 16);
            }
            auto* cwd{reinterpret_cast<std::uint32_t*>(win_chroma)};
#pragma unroll
            for (int j{0}; j < kChromaPer; ++j) {
                const int i{tid + j * kThreads};
                if (i < kChromaItems) cwd[i] = cv[j];
            }
        } else {
            constexpr int kLumaPer{(kXplane + kThreads - 1) / kThreads};
            constexpr int kChromaPer{(kChromaWin * kChromaWin + kThreads - 1) / kThreads};
            std::uint8_t lv[kLumaPer], cb[kChromaPer], cr[kChromaPer];
#pragma unroll
            for (int j{0}; j < kLumaPer; ++j) {
                const int i{tid + j * kThreads};
                if (i < kXplane) {
                    const int gx{min(max(px0 - kHalo + i % kXs, 0), W - 1)};
                    const int gy{min(max(py0 - kHalo + i / kXs, 0), H - 1)};
                    lv[j] = in.luma[static_cast<std::size_t>(gy) * in.luma_pitch + gx];
                }
            }
#pragma unroll
            for (int j{0}; j < kChromaPer; ++j) {
                const int i{tid + j * kThreads};
                if (i < kChromaWin * kChromaWin) {
                    const int jx{min(max(cx0 + i % kChromaWin, 0), cw - 1)};
                    const int jy{min(max(cy0 + i / kChromaWin, 0), ch - 1)};
                    const std::uint8_t* p{in.chroma + static_cast<std::size_t>(jy) * in.chroma_pitch + 2 * jx};
                    cb[j] = p[0];
                    cr[j] = p[1];
                }
            }
#pragma unroll
            for (int j{0}; j < kLumaPer; ++j) {
                const int i{tid + j * kThreads};
                if (i < kXplane) win_luma[i] = lv[j];
            }
#pragma unroll
            for (int j{0}; j < kChromaPer; ++j) {
                const int i{tid + j * kThreads};
                if (i < kChromaWin * kChromaWin) {
                    win_chroma[2 * i] = cb[j];
                    win_chroma[2 * i + 1] = cr[j];
                }
            }
        }
        sm.log2_small[tid] = log2_entry;
        if (tid < 4) sm.net[tid] = net_entry;
#pragma unroll
        for (int k{0}; k < 6; ++k) {
            if (tid == k) sm.pow_lut[k] = make_float2(pow24_factor_c(k), pow24_factor_scale(k));
        }
    }
    tile_sync(bar);
    // Regions whose transform split (and, with net_qf, quant field) the
    // network decided; zero without a network.
    unsigned dmask{0};
#pragma unroll
    for (int ri{0}; ri < 4; ++ri) dmask |= (sm.net[ri] >= 0 ? 1u : 0u) << ri;
    const unsigned qmask{in.net_qf != nullptr ? dmask : 0u};
    // 1b. XYB of every halo pixel from the window, two horizontally adjacent
    // pixels per thread (the row length kXs is even, so a pair never spans
    // two rows, and its float2 stores are 8-byte aligned).
    static_assert(kXs % 2 == 0 && kXplane % 2 == 0, "XYB pairs");
    for (int i2{tid}; i2 < kXplane / 2; i2 += kThreads) {
        const int i{2 * i2};
        const int row{i / kXs};
        const int col{i - row * kXs};
        const int gx0{min(max(px0 - kHalo + col, 0), W - 1)};
        const int gx1{min(max(px0 - kHalo + col + 1, 0), W - 1)};
        const int gy{min(max(py0 - kHalo + row, 0), H - 1)};
        float2 x, y, b;
        xyb_pixel2<kChromaWin>(win_luma[i], win_luma[i + 1], win_chroma, cx0, cy0, gx0, gx1, gy, W, H, sm.pow_lut,
                               x, y, b);
        *reinterpret_cast<float2*>(xyb + i) = x;
        *reinterpret_cast<float2*>(xyb + kXplane + i) = y;
        *reinterpret_cast<float2*>(xyb + 2 * kXplane + i) = b;
    }
    tile_sync(bar);

    if (out.dbg_xyb != nullptr) {
        for (int i{tid}; i < 3 * kTile * kTile; i += kThreads) {
            const int c{i / (kTile * kTile)};
            const int p{i % (kTile * kTile)};
            const int gx{px0 + p % kTile};
            const int gy{py0 + p / kTile};
            if (gx < W && gy < H) {
                out.dbg_xyb[(static_cast<std::size_t>(c) * H + gy) * W + gx] =
                    xyb[c * kXplane + (p / kTile + kHalo) * kXs + p % kTile + kHalo];
            }
        }
    }

    // ---- 2. adaptive quantisation (src/frontend_fused.cu:233-342). A tile
    // whose four regions all take their quant field from the network skips
    // the phase (the branch is uniform over the CTA).
    const float* Y{xyb + kXplane};
    if (qmask != 0xFu) {
        {
            // Pixels (dx, dx + 1) of each cell row in pairs on packed f32x2
            // arithmetic (the division and square root stay scalar); the sum
            // still accumulates in raster order.
            const int ccx{tid & 15};
            const int ccy{tid >> 4};
            const int ix0{ccx * 4 + kHalo};  // even: the float2 loads below are aligned
            float sum{0.0f};
    #pragma unroll
            for (int dy{0}; dy < 4; ++dy) {
                const int iy{ccy * 4 + dy + kHalo};
                const float* C{Y + iy * kXs + ix0};
                const float* U{C - kXs};
                const float* D{C + kXs};
                const float2 c0{*reinterpret_cast<const float2*>(C - 2)};  // ix0-2, ix0-1
                const float2 c1{*reinterpret_cast<const float2*>(C)};      // ix0, ix0+1
                const float2 c2{*reinterpret_cast<const float2*>(C + 2)};  // ix0+2, ix0+3
                const float2 c3{*reinterpret_cast<const float2*>(C + 4)};  // ix0+4, ix0+5
                const float2 up[2]{*reinterpret_cast<const float2*>(U), *reinterpret_cast<const float2*>(U + 2)};
                const float2 dn[2]{*reinterpret_cast<const float2*>(D), *reinterpret_cast<const float2*>(D + 2)};
                const float2 ctr[2]{c1, c2};
                const float2 lft[2]{make_float2(c0.y, c1.x), make_float2(c1.y, c2.x)};
                const float2 rgt[2]{make_float2(c1.y, c2.x), make_float2(c2.y, c3.x)};
    #pragma unroll
                for (int h{0}; h < 2; ++h) {
                    const float2 yv{ctr[h]};
                    const float2 base{__fmul2_rn(
                        f2dup(0.25f), __fadd2_rn(__fadd2_rn(__fadd2_rn(dn[h], up[h]), lft[h]), rgt[h]))};
                    // ratio_gamma<false>(yv + kMatchGammaOffset)
                    float2 v{__fadd2_rn(yv, f2dup(kMatchGammaOffset))};
                    v = make_float2(v.x < 0.0f ? 0.0f : v.x, v.y < 0.0f ? 0.0f : v.y);
                    const float2 v2{__fmul2_rn(v, v)};
                    const float2 num{__ffma2_rn(f2dup(kRatioNumMul), v2, f2dup(kRatioEps))};
                    const float2 den{__ffma2_rn(__fmul2_rn(f2dup(kRatioDenMul), v), v2, f2dup(kRatioVOffset))};
                    const float2 ratio{div2_ratio(den, num)};
                    float2 d{__fmul2_rn(ratio, __fadd2_rn(yv, f2neg(base)))};
                    d = __fmul2_rn(d, d);
                    d = make_float2(fminf(d.x, kDiffLimit), fminf(d.y, kDiffLimit));
                    // Masking square root 0.25 * sqrt(d * mul + offset) (src/adaptive_quant_impl.cuh:57-61).
                    const float2 t{__ffma2_rn(d, f2dup(sc.mask_sqrt_mul), f2dup(kMaskLogOffset))};
                    const float2 m{__fmul2_rn(f2dup(0.25f), make_float2(sqrtf(t.x), sqrtf(t.y)))};
                    sum = sum + m.x;
                    sum = sum + m.y;
                }
            }
            sm.pre[tid] = 0.25f * sum;
        }
        tile_sync(bar);
        // The four eroded cells of each of this warp's 8 blocks (block warp + 8j),
        // one per lane: lane 4j + k holds cell k = (k & 1, k >> 1) of block j's
        // 2x2 cells. Their sum (e0 + e2) + (e1 + e3) is the order in which a
        // 32-lane tree with the cells in lanes 0-3 and zeros elsewhere adds them.
        float ero_sum;
        {
            const int lb{warp + 8 * (lane >> 2)};
            const int k{lane & 3};
            const int lbx{lb & 7};
            const int lby{lb >> 3};
            const float e{erosion_cell(sm.pre, (lbx >> 2) * 8, (lby >> 2) * 8, 2 * (lbx & 3) + (k & 1),
                                       2 * (lby & 3) + (k >> 1), sc.km0, sc.km1, sc.km2, sc.km3)};
            const float s{e + __shfl_down_sync(0xffffffffu, e, 2)};
            ero_sum = s + __shfl_down_sync(0xffffffffu, s, 1);
        }
        for (int lb{warp}; lb < 64; lb += kThreads / 32) {
            const int lbx{lb & 7};
            const int lby{lb >> 3};
            const int gbx{bx0 + lbx};
            const int gby{by0 + lby};
            const float eroded{__shfl_sync(0xffffffffu, ero_sum, 4 * (lb >> 3))};
            if (gbx >= bw || gby >= bh || ((qmask >> region_of_block(lb)) & 1u) != 0) {
                continue;  // warp-uniform
            }
            const int fx{lane & 7};
            // Rows fy and fy + 4 of the block as the two components of packed
            // pairs; each half's tree is the reference's, run on both at once.
            const int fy{lane >> 3};
            const int ix{lbx * 8 + fx + kHalo};
            const int iy{lby * 8 + fy + kHalo};
            const int i0{iy * kXs + ix};
            const int i1{i0 + 4 * kXs};
            const float2 yv{Y[i0], Y[i1]};
            const float2 xv{xyb[i0], xyb[i1]};
            const float2 bv{xyb[2 * kXplane + i0], xyb[2 * kXplane + i1]};
            float2 hf{0.0f, 0.0f};
            if (fx < 7) {
                const float2 d{__fadd2_rn(yv, f2neg(make_float2(Y[i0 + 1], Y[i1 + 1])))};
                hf = __fadd2_rn(hf, make_float2(fminf(kHfValMin, fabsf(d.x)), fminf(kHfValMin, fabsf(d.y))));
            }
            {
                // Row fy + 4 has no lower neighbour in the block when it is 7; its
                // term is then +0, which leaves the non-negative sum unchanged.
                const float2 d{__fadd2_rn(yv, f2neg(make_float2(Y[i0 + kXs], Y[i1 + kXs])))};
                hf = __fadd2_rn(hf, make_float2(fminf(kHfValMin, fabsf(d.x)),
                                                fy + 4 < 7 ? fminf(kHfValMin, fabsf(d.y)) : 0.0f));
            }
            const float2 iny{__fadd2_rn(yv, f2dup(kGammaBias))};
            const float2 gp{__fadd2_rn(ratio_gamma_inv2(__fadd2_rn(iny, f2neg(xv))),
                                       ratio_gamma_inv2(__fadd2_rn(iny, xv)))};
            const float2 pye{__fadd2_rn(__fadd2_rn(yv, f2dup(kBlueOffset)), make_float2(fabsf(xv.x), fabsf(xv.y)))};
            const float2 bd{__fadd2_rn(bv, f2neg(pye))};
            const float2 bp{bv.x > pye.x ? fminf(bd.x, kBlueLimit) : 0.0f,
                            bv.y > pye.y ? fminf(bd.y, kBlueLimit) : 0.0f};
            const float2 red0{warp_tree2(hf)};
            const float2 red1{warp_tree2(gp)};
            const float2 red2{warp_tree2(bp)};
            if (lane == 0) {
                // The block's quant field is finished from these sums by its own
                // thread in step 4e, where most warps are otherwise idle. The
                // eroded sum gets the second half's tree of zeros added, as the
                // per-half reduction did.
                sm.aq_sums[0][lb] = red0.x + red0.y;
                sm.aq_sums[1][lb] = red1.x + red1.y;
                sm.aq_sums[2][lb] = red2.x + red2.y;
                sm.aq_sums[3][lb] = eroded + 0.0f;
            }
        }
    }

    // ---- 3. inverse gaborish, 5x5 with image-border clamping (src/frontend_transform.cu:19-36).
    // Two horizontally adjacent outputs (x even) of four adjacent rows per
    // thread on packed f32x2 arithmetic: each of the eight source rows' six
    // samples x-2..x+3 come in as three aligned float2 loads (the row stride
    // kXs and x + kHalo - 2 are even), shared by the output rows that use
    // them, and operand pair (dx, dy) is {row[x+dx], row[x+1+dx]}. (Four rows
    // instead of two: 14.1K -> 12.8K cycles per tile for the phase.)
    static_assert(kXs % 2 == 0 && kHalo % 2 == 0, "gaborish pairs");
    for (int i8{tid}; i8 < 3 * kTile * kTile / 8; i8 += kThreads) {
        const int c{i8 >> 9};
        const int p8{i8 & 511};
        const int x{2 * (p8 & 31)};
        const int y0{4 * (p8 >> 5)};
        const float* P{xyb + c * kXplane + y0 * kXs + x};  // sample (x - 2, y0 - 2)
        float2 row[8][5];  // row[r][dx + 2] of source row y0 - 2 + r
#pragma unroll
        for (int r{0}; r < 8; ++r) {
            const float2 a{*reinterpret_cast<const float2*>(P + r * kXs)};
            const float2 b{*reinterpret_cast<const float2*>(P + r * kXs + 2)};
            const float2 d{*reinterpret_cast<const float2*>(P + r * kXs + 4)};
            row[r][0] = a;
            row[r][1] = make_float2(a.y, b.x);
            row[r][2] = b;
            row[r][3] = make_float2(b.y, d.x);
            row[r][4] = d;
        }
#pragma unroll
        for (int h{0}; h < 4; ++h) {
            auto at = [&](int dx, int dy) { return row[h + dy + 2][dx + 2]; };
            auto add = [](float2 u, float2 v) { return __fadd2_rn(u, v); };
            const float2 e{add(add(add(at(-1, 0), at(1, 0)), at(0, -1)), at(0, 1))};
            const float2 r2{add(add(add(at(-2, 0), at(2, 0)), at(0, -2)), at(0, 2))};
            const float2 dg{add(add(add(at(-1, -1), at(1, -1)), at(-1, 1)), at(1, 1))};
            const float2 l8{add(add(add(add(add(add(add(at(-2, -1), at(2, -1)), at(-2, 1)), at(2, 1)), at(-1, -2)),
                                        at(1, -2)), at(-1, 2)), at(1, 2))};
            const float2 d4{add(add(add(at(-2, -2), at(2, -2)), at(-2, 2)), at(2, 2))};
            float2 sv{__fmul2_rn(f2dup(kGabC), at(0, 0))};
            sv = __ffma2_rn(f2dup(kGabEdge), e, sv);
            sv = __ffma2_rn(f2dup(kGabEdge2), r2, sv);
            sv = __ffma2_rn(f2dup(kGabDiag), dg, sv);
            sv = __ffma2_rn(f2dup(kGabKnight), l8, sv);
            sv = __ffma2_rn(f2dup(kGabDiag2), d4, sv);
            *reinterpret_cast<float2*>(shp + c * kSplane + (y0 + h) * kSs + x) = sv;
        }
    }
    tile_sync(bar);

    if (out.dbg_sharp != nullptr) {
        for (int i{tid}; i < 3 * kTile * kTile; i += kThreads) {
            const int c{i >> 12};
            const int p{i & 4095};
            const int gx{px0 + (p & 63)};
            const int gy{py0 + (p >> 6)};
            if (gx < W && gy < H) {
                out.dbg_sharp[(static_cast<std::size_t>(c) * H + gy) * W + gx] =
                    shp[c * kSplane + (p >> 6) * kSs + (p & 63)];
            }
        }
    }

    // ---- 4. transform selection on the sharpened Y (src/transform_select.cu:134-262).
    const float* SY{shp + kSplane};
    float* rows{smem};             // region A reused: row-pass scratch
    float* cdist{smem + 4608};     // per-coefficient distortion contributions
    float* crate{smem + 9216};     // per-coefficient rate contributions
    const float qg{sc.qgsf_select};
    // Regions inside the image that the network did not decide need the RD
    // costs; when there are none the cost passes are skipped altogether.
    unsigned inimg{0};
#pragma unroll
    for (int ri{0}; ri < 4; ++ri) {
        inimg |= (bx0 + 4 * (ri & 1) < bw && by0 + 4 * (ri >> 1) < bh ? 1u : 0u) << ri;
    }
    if ((inimg & ~dmask) != 0u) {
        // 4a. DCT8 candidates: one per block inside the image.
        for (int k{tid}; k < 512; k += kThreads) {
            const int lb{k >> 3};
            const int r{k & 7};
            const int lbx{lb & 7};
            const int lby{lb >> 3};
            if (bx0 + lbx < bw && by0 + lby < bh && ((dmask >> region_of_block(lb)) & 1u) == 0) {
                row_pass<8, 0, 8, true>(SY + (lby * 8 + r) * kSs + lbx * 8, rows + lb * 72 + r);
            }
        }
        tile_sync(bar);
        for (int k{tid}; k < 512; k += kThreads) {
            const int lb{k >> 3};
            const int fx{k & 7};
            if (bx0 + (lb & 7) < bw && by0 + (lb >> 3) < bh &&
                ((dmask >> region_of_block(lb)) & 1u) == 0) {
                sel_col<8, 0, 8>(rows + lb * 72 + fx * 9, cdist + lb * 72 + fx * 9,
                                 crate + lb * 72 + fx * 9, fx, qg, tb.sel_weight, tb.log2_1p, sm.log2_small);
            }
        }
        tile_sync(bar);
        // Distortion and rate ride one packed pair through each step.
#pragma unroll 2
        for (int lb{warp}; lb < 64; lb += kThreads / 32) {
            if (bx0 + (lb & 7) < bw && by0 + (lb >> 3) < bh &&
                ((dmask >> region_of_block(lb)) & 1u) == 0) {
                const int i0{lb * 72 + (lane >> 3) * 9 + (lane & 7)};
                const int i1{lb * 72 + ((lane + 32) >> 3) * 9 + (lane & 7)};
                const float2 DR{warp_tree2(
                    __fadd2_rn(make_float2(cdist[i0], crate[i0]), make_float2(cdist[i1], crate[i1])))};
                if (lane == 0) {
                    sm.cost8[lb] = 64.0f * DR.x + kSelectLambda * DR.y;
                }
            }
        }
        // 4b. DCT16 candidates: the 16 quads of the tile that fit in the image.
        // Their row pass writes only the row scratch, which the DCT8
        // reduction above does not read, so it shares that phase.
        for (int k{tid}; k < 256; k += kThreads) {
            const int qd{k >> 4};
            const int r{k & 15};
            const int qx{qd & 3};
            const int qy{qd >> 2};
            if (bx0 + 2 * qx + 2 <= bw && by0 + 2 * qy + 2 <= bh &&
                ((dmask >> (((qy >> 1) << 1) | (qx >> 1))) & 1u) == 0) {
                row_pass<16, 0, 16, true>(SY + (qy * 16 + r) * kSs + qx * 16, rows + qd * 272 + r);
            }
        }
        tile_sync(bar);
        for (int k{tid}; k < 256; k += kThreads) {
            const int qd{k >> 4};
            const int fx{k & 15};
            if (bx0 + 2 * (qd & 3) + 2 <= bw && by0 + 2 * (qd >> 2) + 2 <= bh &&
                ((dmask >> (((qd >> 3) << 1) | ((qd & 3) >> 1))) & 1u) == 0) {
                sel_col<16, 0, 16>(rows + qd * 272 + fx * 17, cdist + qd * 272 + fx * 17,
                                   crate + qd * 272 + fx * 17, fx, qg, tb.sel_weight + 1024,
                                   tb.log2_1p, sm.log2_small);
            }
        }
        tile_sync(bar);
        for (int qd{warp}; qd < 16; qd += kThreads / 32) {
            if (bx0 + 2 * (qd & 3) + 2 <= bw && by0 + 2 * (qd >> 2) + 2 <= bh &&
                ((dmask >> (((qd >> 3) << 1) | ((qd & 3) >> 1))) & 1u) == 0) {
                // Distortion (x) and rate (y) as packed pairs, each in the
                // host twin's order.
                float2 p[8];
#pragma unroll
                for (int j{0}; j < 8; ++j) {
                    const int t{lane + 32 * j};
                    const int at{qd * 272 + (t >> 4) * 17 + (t & 15)};
                    p[j] = make_float2(cdist[at], crate[at]);
                }
#pragma unroll
                for (int j{0}; j < 4; ++j) p[j] = __fadd2_rn(p[j], p[j + 4]);
                p[0] = __fadd2_rn(p[0], p[2]);
                p[1] = __fadd2_rn(p[1], p[3]);
                const float2 DR{warp_tree2(__fadd2_rn(p[0], p[1]))};
                if (lane == 0) {
                    sm.cost16[qd] = 256.0f * DR.x + kSelectLambda * DR.y;
                }
            }
        }
        // 4c. DCT32 candidates: the 4 regions of the tile that fit in the image.
        // Their row pass shares the DCT16 reduction's phase (disjoint
        // scratch).
        for (int k{tid}; k < 256; k += kThreads) {
            const int ri{k >> 6};
            const int r{k & 31};
            const bool hi{(k & 32) != 0};
            const int rx{ri & 1};
            const int ry{ri >> 1};
            if (bx0 + 4 * rx + 4 <= bw && by0 + 4 * ry + 4 <= bh && ((dmask >> ri) & 1u) == 0) {
                const float* src{SY + (ry * 32 + r) * kSs + rx * 32};
                float* dst{rows + ri * 1056 + r};
                if (hi) {
                    row_pass<32, 16, 32, true>(src, dst);
                } else {
                    row_pass<32, 0, 16, true>(src, dst);
                }
            }
        }
        tile_sync(bar);
        for (int k{tid}; k < 256; k += kThreads) {
            const int ri{k >> 6};
            const int fx{k & 31};
            const bool hi{(k & 32) != 0};
            if (bx0 + 4 * (ri & 1) + 4 <= bw && by0 + 4 * (ri >> 1) + 4 <= bh &&
                ((dmask >> ri) & 1u) == 0) {
                const float* src{rows + ri * 1056 + fx * 33};
                float* cd{cdist + ri * 1056 + fx * 33};
                float* cr{crate + ri * 1056 + fx * 33};
                if (hi) {
                    sel_col<32, 16, 32>(src, cd, cr, fx, qg, tb.sel_weight + 2048, tb.log2_1p, sm.log2_small);
                } else {
                    sel_col<32, 0, 16>(src, cd, cr, fx, qg, tb.sel_weight + 2048, tb.log2_1p, sm.log2_small);
                }
            }
        }
        tile_sync(bar);
        if (warp < 4) {
            const int ri{warp};
            if (bx0 + 4 * (ri & 1) + 4 <= bw && by0 + 4 * (ri >> 1) + 4 <= bh &&
                ((dmask >> ri) & 1u) == 0) {
                // Distortion (x) and rate (y) as packed pairs, each in the
                // host twin's order.
                float2 p[8];
#pragma unroll
                for (int j{0}; j < 8; ++j) {
                    float2 dr{0.0f, 0.0f};
#pragma unroll
                    for (int m{0}; m < 4; ++m) {
                        const int e{lane + 32 * j + 256 * m};
                        const int at{ri * 1056 + (e >> 5) * 33 + (e & 31)};
                        dr = __fadd2_rn(dr, make_float2(cdist[at], crate[at]));
                    }
                    p[j] = dr;
                }
#pragma unroll
                for (int j{0}; j < 4; ++j) p[j] = __fadd2_rn(p[j], p[j + 4]);
                p[0] = __fadd2_rn(p[0], p[2]);
                p[1] = __fadd2_rn(p[1], p[3]);
                const float2 DR{warp_tree2(__fadd2_rn(p[0], p[1]))};
                if (lane == 0) {
                    sm.cost32[ri] = 1024.0f * DR.x + kSelectLambda * DR.y;
                }
            }
        }
    }
    // 4d. RD decision per region (src/transform_select_impl.cuh:130-201), by
    // lane 0 of warp ri, which wrote cost32[ri] itself (the DCT8 and DCT16
    // costs are older than the last barrier).
    if (warp < 4 && lane == 0) {
        const int ri{warp};
        const int rlx{(ri & 1) * 4};
        const int rly{(ri >> 1) * 4};
        const int rbx{bx0 + rlx};
        const int rby{by0 + rly};
        if (((dmask >> ri) & 1u) != 0) {
            // Network split of a full region: class 0 is one DCT32, class
            // 1 + m has quadrant q as four DCT8 when bit q of m is set, else
            // as one DCT16.
            const int cls{sm.net[ri]};
            for (int dy{0}; dy < 4; ++dy) {
                for (int dx{0}; dx < 4; ++dx) {
                    const int q{(dy >> 1) * 2 + (dx >> 1)};
                    signed char a;
                    if (cls == 0) {
                        a = (dx == 0 && dy == 0) ? 32 : 0;
                    } else if ((((cls - 1) >> q) & 1) != 0) {
                        a = 8;
                    } else {
                        a = ((dx & 1) == 0 && (dy & 1) == 0) ? 16 : 0;
                    }
                    sm.acs[(rly + dy) * 8 + rlx + dx] = a;
                }
            }
        } else if (rbx < bw && rby < bh) {
            constexpr float kInf{1.0e30f};
            const bool fit32{rbx + 4 <= bw && rby + 4 <= bh};
            const float c32{fit32 ? sm.cost32[ri] : kInf};
            float split{0.0f};
            int choice[2][2];
            for (int qy{0}; qy < 2; ++qy) {
                for (int qx{0}; qx < 2; ++qx) {
                    const int bx{rbx + 2 * qx};
                    const int by{rby + 2 * qy};
                    float sum8{0.0f};
                    bool any{false};
                    for (int dy{0}; dy < 2; ++dy) {
                        for (int dx{0}; dx < 2; ++dx) {
                            if (bx + dx < bw && by + dy < bh) {
                                sum8 = sum8 + sm.cost8[(rly + 2 * qy + dy) * 8 + rlx + 2 * qx + dx];
                                any = true;
                            }
                        }
                    }
                    if (!any) {
                        choice[qy][qx] = -1;
                        continue;
                    }
                    const bool fit16{bx + 2 <= bw && by + 2 <= bh};
                    const float c16{fit16 ? sm.cost16[((rly >> 1) + qy) * 4 + (rlx >> 1) + qx] : kInf};
                    if (fit16 && c16 <= sum8 + kSelectSplitEps) {
                        choice[qy][qx] = 16;
                        split = split + c16;
                    } else {
                        choice[qy][qx] = 8;
                        split = split + sum8;
                    }
                }
            }
            if (fit32 && c32 <= split + kSelectSplitEps) {
                for (int dy{0}; dy < 4; ++dy) {
                    for (int dx{0}; dx < 4; ++dx) {
                        sm.acs[(rly + dy) * 8 + rlx + dx] = (dx == 0 && dy == 0) ? 32 : 0;
                    }
                }
            } else {
                for (int qy{0}; qy < 2; ++qy) {
                    for (int qx{0}; qx < 2; ++qx) {
                        const int ch{choice[qy][qx]};
                        if (ch < 0) {
                            continue;
                        }
                        for (int dy{0}; dy < 2; ++dy) {
                            for (int dx{0}; dx < 2; ++dx) {
                                const int l{(rly + 2 * qy + dy) * 8 + rlx + 2 * qx + dx};
                                if (ch == 16) {
                                    sm.acs[l] = (dx == 0 && dy == 0) ? 16 : 0;
                                } else if (rbx + 2 * qx + dx < bw && rby + 2 * qy + dy < bh) {
                                    sm.acs[l] = 8;
                                }
                            }
                        }
                    }
                }
            }
        }
    }
    // Warps 4-7 meanwhile clear the non-zero counters and CfL sums and finish
    // each block's quant field from its AQ sums.
    if (tid >= 128) {
        for (int i{tid - 128}; i < 192; i += 128) {
            sm.nz[i >> 6][i & 63] = 0;
            sm.cfl[i >> 6][i & 63] = 0.0f;  // blocks that are not first blocks add zero
        }
    }
    if (tid >= 128 && tid < 192) {
        // Quant field of block lb from its AQ sums (src/frontend_fused.cu:177-201).
        const int lb{tid - 128};
        if (((qmask >> region_of_block(lb)) & 1u) != 0) {
            sm.qf[lb] = in.net_qf[static_cast<std::size_t>(by0 + (lb >> 3)) * bw + bx0 + (lb & 7)];
        } else if (bx0 + (lb & 7) < bw && by0 + (lb >> 3) < bh) {
            const float hf_sum{sm.aq_sums[0][lb]};
            const float gamma_overall{sm.aq_sums[1][lb] * (0.5f / 64.0f)};
            float blue_sum{sm.aq_sums[2][lb]};
            const float aq{sm.aq_sums[3][lb]};
            if (blue_sum >= 32.0f * kBlueLimit) {
                blue_sum = 64.0f * kBlueLimit - blue_sum;
            }
            if (blue_sum >= kBlueMaxLimit * kBlueLimit) {
                blue_sum = kBlueMaxLimit * kBlueLimit;
            }
            float ov{compute_mask(aq)};
            ov = ov + jx_fma(hf_sum, kHfMul, kHfAdd);
            ov = jx_fma(kGammaLogMul, jx_log2(gamma_overall), ov);
            ov = jx_fma(blue_sum, kBlueMul, ov);
            const float qval{jx_fma(jx_exp(ov), sc.mul_pb, sc.add_pb)};
            int qi{static_cast<int>(jx_fma(qval, sc.inv_global_scale, 0.5f))};
            qi = qi < 1 ? 1 : (qi > kQuantMax ? kQuantMax : qi);
            sm.qf[lb] = qi;
        }
    }
    tile_sync(bar);
    if (out.dbg_cost != nullptr) {
        for (int lb{tid}; lb < 64; lb += kThreads) {
            const int lbx{lb & 7};
            const int lby{lb >> 3};
            if (bx0 + lbx < bw && by0 + lby < bh) {
                const std::size_t at{static_cast<std::size_t>(by0 + lby) * bw + bx0 + lbx};
                out.dbg_cost[at] = sm.cost8[lb];
                out.dbg_cost[nblocks + at] =
                    ((lbx | lby) & 1) == 0 ? sm.cost16[(lby >> 1) * 4 + (lbx >> 1)] : 0.0f;
                out.dbg_cost[2 * static_cast<std::size_t>(nblocks) + at] =
                    ((lbx | lby) & 3) == 0 ? sm.cost32[(lby >> 2) * 2 + (lbx >> 2)] : 0.0f;
            }
        }
    }
    // 4e. first-block list (DCT32 first, then DCT16, then DCT8, each in raster
    // order) with each entry's row-pass scratch offset, and the covering owner
    // of every block; warp 0, two blocks per lane.
    if (warp == 0) {
        int side[2];
        bool in[2];
#pragma unroll
        for (int h{0}; h < 2; ++h) {
            const int lb{lane + 32 * h};
            in[h] = bx0 + (lb & 7) < bw && by0 + (lb >> 3) < bh;
            side[h] = in[h] ? sm.acs[lb] : 0;
            // The owner is the one first block within 3 blocks up and left
            // whose transform reaches this block.
            int own{255};
            for (int dy{0}; dy < 4 && in[h]; ++dy) {
                for (int dx{0}; dx < 4; ++dx) {
                    const int fx{(lb & 7) - dx};
                    const int fy{(lb >> 3) - dy};
                    if (fx < 0 || fy < 0) continue;
                    const int s{sm.acs[fy * 8 + fx] >> 3};
                    if (s > dx && s > dy) own = fy * 8 + fx;
                }
            }
            sm.owner[lb] = static_cast<unsigned char>(own);
        }
        int at{0};
        int off{0};
        const unsigned below{(1u << lane) - 1u};
#pragma unroll
        for (int g{0}; g < 3; ++g) {
            const int s{32 >> g};
            const int step{s * (s + (s == 32 ? 4 : 1))};  // row strides 36, 17, 9 (kDrowsStride)
            const unsigned m0{__ballot_sync(0xffffffffu, side[0] == s)};
            const unsigned m1{__ballot_sync(0xffffffffu, side[1] == s)};
            const int c0{__popc(m0)};
            if (side[0] == s) {
                const int r{at + __popc(m0 & below)};
                sm.fb_list[r] = static_cast<unsigned char>(lane);
                sm.fb_off[r] = off + (r - at) * step;
            }
            if (side[1] == s) {
                const int r{at + c0 + __popc(m1 & below)};
                sm.fb_list[r] = static_cast<unsigned char>(lane + 32);
                sm.fb_off[r] = off + (r - at) * step;
            }
            const int cnt{c0 + __popc(m1)};
            if (lane == 0) {
                if (g == 0) sm.n32 = cnt;
                if (g == 1) sm.n16 = cnt;
                if (g == 2) sm.n8 = cnt;
            }
            at += cnt;
            off += cnt * step;
        }
    }
    tile_sync(bar);

    // ---- 5. variable DCT of X, Y, B -> FP16 coefficients (src/frontend_transform.cu:190-266).
    // The three channels' row passes run in one phase (each channel has its
    // own row scratch in region A), then their column passes in another; the
    // FP16 coefficients of channel c go over sharpened plane c, which its row
    // pass has finished reading.
    __half* coef{reinterpret_cast<__half*>(shp)};  // [3][64 blocks][kCoefBlock], channel stride kCoefStride
    const int n32{sm.n32};
    const int n16{sm.n16};
    const int n8{sm.n8};
    const int t32{64 * n32};
    const int t16{t32 + 16 * n16};
    const int tall{t16 + 8 * n8};
    for (int k3{tid}; k3 < 3 * tall; k3 += kThreads) {
        const int c{k3 >= 2 * tall ? 2 : (k3 >= tall ? 1 : 0)};
        const int k{k3 - c * tall};
        const float* P{shp + c * kSplane};
        float* drows{smem + c * kDrowsChannel};
        if (k < t32) {
            const int f{k >> 6};
            const int lb{sm.fb_list[f]};
            const int r{k & 31};
            const float* src{P + ((lb >> 3) * 8 + r) * kSs + (lb & 7) * 8};
            float* dst{drows + sm.fb_off[f] + r};
            if (k & 32) {
                row_pass<32, 16, 32, false>(src, dst);
            } else {
                row_pass<32, 0, 16, false>(src, dst);
            }
        } else if (k < t16) {
            const int f{n32 + ((k - t32) >> 4)};
            const int lb{sm.fb_list[f]};
            const int r{(k - t32) & 15};
            row_pass<16, 0, 16, false>(P + ((lb >> 3) * 8 + r) * kSs + (lb & 7) * 8, drows + sm.fb_off[f] + r);
        } else {
            const int f{n32 + n16 + ((k - t16) >> 3)};
            const int lb{sm.fb_list[f]};
            const int r{(k - t16) & 7};
            row_pass<8, 0, 8, false>(P + ((lb >> 3) * 8 + r) * kSs + (lb & 7) * 8, drows + sm.fb_off[f] + r);
        }
    }
    tile_sync(bar);
    for (int k3{tid}; k3 < 3 * tall; k3 += kThreads) {
        const int c{k3 >= 2 * tall ? 2 : (k3 >= tall ? 1 : 0)};
        const int k{k3 - c * tall};
        const float* drows{smem + c * kDrowsChannel};
        __half* cc{coef + c * kCoefStride};
        if (k < t32) {
            const int f{k >> 6};
            const int lb{sm.fb_list[f]};
            const int fx{k & 31};
            const float* src{drows + sm.fb_off[f] + fx * kDrowsStride<32>};
            if (k & 32) {
                dct_col<32, 16, 32>(src, cc, fx, lb & 7, lb >> 3);
            } else {
                dct_col<32, 0, 16>(src, cc, fx, lb & 7, lb >> 3);
            }
        } else if (k < t16) {
            const int f{n32 + ((k - t32) >> 4)};
            const int lb{sm.fb_list[f]};
            const int fx{(k - t32) & 15};
            dct_col<16, 0, 16>(drows + sm.fb_off[f] + fx * 17, cc, fx, lb & 7, lb >> 3);
        } else {
            const int f{n32 + n16 + ((k - t16) >> 3)};
            const int lb{sm.fb_list[f]};
            const int fx{(k - t16) & 7};
            dct_col<8, 0, 8>(drows + sm.fb_off[f] + fx * 9, cc, fx, lb & 7, lb >> 3);
        }
    }
    tile_sync(bar);

    if (out.dbg_coeff != nullptr) {
        for (int i{tid}; i < 3 * 4096; i += kThreads) {
            const int c{i >> 12};
            const int lb{(i >> 6) & 63};
            const int gbx{bx0 + (lb & 7)};
            const int gby{by0 + (lb >> 3)};
            if (gbx < bw && gby < bh) {
                out.dbg_coeff[static_cast<std::size_t>(c) * nblocks * 64 +
                              (static_cast<std::size_t>(gby) * bw + gbx) * 64 + (i & 63)] =
                    __half_as_ushort(coef[c * kCoefStride + lb * kCoefBlock + (i & 63)]);
            }
        }
    }

    // ---- 6. chroma from luma over the tile (src/frontend_quantize.cu:49-117),
    // and DC from the low-frequency corners (src/frontend_quantize.cu:180-200,
    // src/vardct_layout.h:88-111), which needs no CfL result. Warps 0-5 take
    // the (first block, sum kind) pairs round-robin, the largest transforms
    // first, each sum across the warp (cfl_sum_warp). Warps 6-7: one 8x8 DC
    // position per thread.
    if (tid < 192) {
        const int nfb{sm.n32 + sm.n16 + sm.n8};
        for (int t{warp}; t < 3 * nfb; t += 6) {
            const int i{t / 3};
            const int which{t - 3 * i};
            const int lb{sm.fb_list[i]};
            const float v{i < sm.n32 ? cfl_sum_kind<32>(coef, lb, which, lane)
                                     : (i < sm.n32 + sm.n16 ? cfl_sum_kind<16>(coef, lb, which, lane)
                                                            : cfl_sum_kind<8>(coef, lb, which, lane))};
            if (lane == 0) sm.cfl[which][lb] = v;
        }
    } else if (tid >= 192) {
        const int p{tid - 192};
        const int f{sm.owner[p]};
        if (bx0 + (p & 7) < bw && by0 + (p >> 3) < bh) {
            const int n{sm.acs[f]};
            const int m{n >> 3};
            const int ox{(p & 7) - (f & 7)};
            const int oy{(p >> 3) - (f >> 3)};
            float dcv[3];
            if (m == 1) {
                for (int c{0}; c < 3; ++c) {
                    dcv[c] = __half2float(coef[c * kCoefStride + f * kCoefBlock]);
                }
            } else if (m == 2) {
                llf_to_dc<2>(coef, f, ox, oy, tb.llf_basis, dcv);
            } else {
                llf_to_dc<4>(coef, f, ox, oy, tb.llf_basis + 16, dcv);
            }
            const float dcq_x{4096.0f * sc.dc_scale};
            const float dcq_y{512.0f * sc.dc_scale};
            const float dcq_b{256.0f * sc.dc_scale};
            const std::size_t blk{static_cast<std::size_t>(by0 + (p >> 3)) * bw + bx0 + (p & 7)};
            const int qdy{static_cast<int>(lrintf(dcv[1] * dcq_y))};
            const float ydr{static_cast<float>(qdy) / dcq_y};
            out.dc[nblocks + blk] = qdy;
            out.dc[blk] = static_cast<int>(lrintf(dcv[0] * dcq_x));
            out.dc[2 * static_cast<std::size_t>(nblocks) + blk] = static_cast<int>(lrintf((dcv[2] - ydr) * dcq_b));
        }
    }
    tile_sync(bar);
    // The tile's maps: every warp reduces the 64 partials itself (the same
    // tree, so the same maps on every warp) instead of waiting at one more
    // barrier for warp 0 to do it. The trees leave the sums in lane 0, which
    // hands its maps to the other lanes.
    int cfl_mx;
    int cfl_mb;
    {
        const float2 sxy_yy{warp_tree2(__fadd2_rn(make_float2(sm.cfl[0][lane], sm.cfl[1][lane]),
                                                  make_float2(sm.cfl[0][lane + 32], sm.cfl[1][lane + 32])))};
        const float sxy{sxy_yy.x};
        const float syy{sxy_yy.y};
        const float sby{warp_tree(sm.cfl[2][lane] + sm.cfl[2][lane + 32])};
        // The reference divides the float sums in double and rounds the
        // quotient to float; with 53 >= 2 * 24 + 2 significand bits that
        // double rounding equals float division's single rounding
        // (Figueroa, "When is double rounding innocuous?", SIGNUM 1995),
        // so the float quotient is the same value.
        const float fx{syy > 0.0f ? sxy / syy : 0.0f};
        const float fb{syy > 0.0f ? sby / syy : 0.0f};
        int mx{static_cast<int>(lrintf(fx * static_cast<float>(kCflColorFactor)))};
        int mb{static_cast<int>(lrintf(fb * static_cast<float>(kCflColorFactor)))};
        cfl_mx = __shfl_sync(0xffffffffu, mx < -128 ? -128 : (mx > 127 ? 127 : mx), 0);
        cfl_mb = __shfl_sync(0xffffffffu, mb < -128 ? -128 : (mb > 127 ? 127 : mb), 0);
        if (tid == 0) {
            const int tile{ty * ((W + kTile - 1) / kTile) + tx};
            out.ytox[tile] = static_cast<std::int8_t>(cfl_mx);
            out.ytob[tile] = static_cast<std::int8_t>(cfl_mb);
        }
    }

    // ---- 7. quantisation (src/frontend_quantize.cu:125-201).
    const float ytox{static_cast<float>(cfl_mx) * kCflColorScale};
    const float ytob{jx_fma(static_cast<float>(cfl_mb), kCflColorScale, kCflBaseB)};
    const std::size_t cplane{static_cast<std::size_t>(nblocks) * 64};
    // Four adjacent slots (raw indices 4m .. 4m + 3, which lie in one row of
    // their block: every row is 8, 16 or 32 long) per thread: lanes 0-15 of a
    // warp's iteration take the 64 slots of one tile block, lanes 16-31 those
    // of the next, so the block's setup serves four slots per lane, weights
    // move as 16-byte loads and outputs as 8-byte stores.
    static_assert(kThreads % 32 == 0 && 1024 % kThreads == 0, "two tile blocks per warp iteration");
    for (int k4{tid}; k4 < 1024; k4 += kThreads) {  // 4 uniform iterations per warp
        const int k{4 * k4};
        const int lb{k >> 6};
        const int slot{k & 63};
        const int lbx{lb & 7};
        const int lby{lb >> 3};
        const bool inside{bx0 + lbx < bw && by0 + lby < bh};
        const int f{inside ? static_cast<int>(sm.owner[lb]) : -1};
        std::int16_t ax[4]{0, 0, 0, 0};
        std::int16_t ay[4]{0, 0, 0, 0};
        std::int16_t ab[4]{0, 0, 0, 0};
        if (inside) {
            const int n{sm.acs[f]};
            const int side{n >> 3};
            const int lrow{side == 1 ? 3 : (side == 2 ? 4 : 5)};  // log2(n)
            const int q{(lby - (f >> 3)) * side + lbx - (f & 7)};
            const int raw{q * 64 + slot};  // a multiple of 4
            const bool llf_row{(raw >> lrow) < side};
            const int col{raw & (n - 1)};
            if (!(llf_row && col + 3 < side)) {
                const int si{n == 8 ? 0 : (n == 16 ? 1 : 2)};
                const float* wt{tb.dequant + si * 3072};
                const float qgsf{static_cast<float>(sm.qf[f]) * sc.gsf};
                const int ci{lb * kCoefBlock + slot};
                auto load4 = [&](const __half* plane, float (&v)[4]) {
                    const float2 lo{__half22float2(*reinterpret_cast<const __half2*>(plane + ci))};
                    const float2 hi{__half22float2(*reinterpret_cast<const __half2*>(plane + ci + 2))};
                    v[0] = lo.x;
                    v[1] = lo.y;
                    v[2] = hi.x;
                    v[3] = hi.y;
                };
                float xr[4], yr[4], br[4];
                load4(coef, xr);
                load4(coef + kCoefStride, yr);
                load4(coef + 2 * kCoefStride, br);
                const float4 wx4{*reinterpret_cast<const float4*>(wt + raw)};
                const float4 wy4{*reinterpret_cast<const float4*>(wt + 1024 + raw)};
                const float4 wb4{*reinterpret_cast<const float4*>(wt + 2048 + raw)};
                const float4 ix4{*reinterpret_cast<const float4*>(wt + kDequantInv + raw)};
                const float4 iy4{*reinterpret_cast<const float4*>(wt + kDequantInv + 1024 + raw)};
                const float4 ib4{*reinterpret_cast<const float4*>(wt + kDequantInv + 2048 + raw)};
                const float wx[4]{wx4.x, wx4.y, wx4.z, wx4.w};
                const float wy[4]{wy4.x, wy4.y, wy4.z, wy4.w};
                const float wb[4]{wb4.x, wb4.y, wb4.z, wb4.w};
                const float ix[4]{ix4.x, ix4.y, ix4.z, ix4.w};
                const float iy[4]{iy4.x, iy4.y, iy4.z, iy4.w};
                const float ib[4]{ib4.x, ib4.y, ib4.z, ib4.w};
#pragma unroll
                for (int h{0}; h < 4; ++h) {
                    if (llf_row && col + h < side) continue;  // an LLF slot
                    const int qy{quantize(yr[h], qgsf, wy[h], iy[h])};
                    // A zero Y quantum reconstructs to a signed zero, and
                    // fma(-m, +-0, v) equals v up to the sign of a zero
                    // result, which quantises to 0 either way.
                    const float yq{qy == 0 ? 0.0f : (static_cast<float>(qy) * wy[h]) / qgsf};
                    ax[h] = static_cast<std::int16_t>(quantize(jx_fma(-ytox, yq, xr[h]), qgsf, wx[h], ix[h]));
                    ay[h] = static_cast<std::int16_t>(qy);
                    ab[h] = static_cast<std::int16_t>(quantize(jx_fma(-ytob, yq, br[h]), qgsf, wb[h], ib[h]));
                }
            }
            const std::size_t g{(static_cast<std::size_t>(by0 + lby) * bw + bx0 + lbx) * 64 + slot};
            *reinterpret_cast<short4*>(out.ac + g) = make_short4(ax[0], ax[1], ax[2], ax[3]);
            *reinterpret_cast<short4*>(out.ac + cplane + g) = make_short4(ay[0], ay[1], ay[2], ay[3]);
            *reinterpret_cast<short4*>(out.ac + 2 * cplane + g) = make_short4(ab[0], ab[1], ab[2], ab[3]);
        }
        // Non-zero counts per first block: each half-warp's 64 slots are one
        // tile block, so lanes 0 and 16 add their half's counts.
        auto nonzero = [](const std::int16_t (&v)[4]) {
            return static_cast<unsigned>((v[0] != 0) + (v[1] != 0) + (v[2] != 0) + (v[3] != 0));
        };
        const unsigned lo_half{lane < 16 ? 1u : 0u};
        const unsigned nx{nonzero(ax)};
        const unsigned ny{nonzero(ay)};
        const unsigned nbz{nonzero(ab)};
        const unsigned cx_lo{__reduce_add_sync(0xffffffffu, lo_half * nx)};
        const unsigned cx_hi{__reduce_add_sync(0xffffffffu, (1u - lo_half) * nx)};
        const unsigned cy_lo{__reduce_add_sync(0xffffffffu, lo_half * ny)};
        const unsigned cy_hi{__reduce_add_sync(0xffffffffu, (1u - lo_half) * ny)};
        const unsigned cb_lo{__reduce_add_sync(0xffffffffu, lo_half * nbz)};
        const unsigned cb_hi{__reduce_add_sync(0xffffffffu, (1u - lo_half) * nbz)};
        if ((lane & 15) == 0 && f >= 0) {
            const unsigned cx{lo_half ? cx_lo : cx_hi};
            const unsigned cy{lo_half ? cy_lo : cy_hi};
            const unsigned cb{lo_half ? cb_lo : cb_hi};
            if (cx) atomicAdd(&sm.nz[0][f], static_cast<int>(cx));
            if (cy) atomicAdd(&sm.nz[1][f], static_cast<int>(cy));
            if (cb) atomicAdd(&sm.nz[2][f], static_cast<int>(cb));
        }
    }
    tile_sync(bar);

    // ---- 8. side information.
    for (int k{tid}; k < 64; k += kThreads) {
        const int lb{k};
        const int gbx{bx0 + (lb & 7)};
        const int gby{by0 + (lb >> 3)};
        if (gbx >= bw || gby >= bh) {
            continue;
        }
        const std::size_t blk{static_cast<std::size_t>(gby) * bw + gbx};
        const int f{sm.owner[lb]};
        const int n{sm.acs[f]};
        const int covered{(n >> 3) * (n >> 3)};
        const int l2{n == 16 ? 2 : (n == 32 ? 4 : 0)};
        for (int c{0}; c < 3; ++c) {
            const int nz{sm.nz[c][f]};
            out.nzn[c * static_cast<std::size_t>(nblocks) + blk] =
                static_cast<std::uint8_t>((nz + covered - 1) >> l2);
            out.nzc[c * static_cast<std::size_t>(nblocks) + blk] =
                static_cast<std::uint16_t>(f == lb ? nz : 0);
        }
        out.acs[blk] = sm.acs[lb];
        out.qf[blk] = sm.qf[lb];
    }
}

// Two tiles per CTA, one per half, each half on its own named barrier:
// tiles (2 blockIdx.x, blockIdx.y) and (2 blockIdx.x + 1, blockIdx.y), or with
// kOrdered entries 2b and 2b + 1 of in.tile_order for CTA b. The two tiles
// start together and run the same code at about the same time, so each
// instruction fetch serves the warps of both; as two CTAs per SM (each one
// tile at its own point of the long unrolled code) the tiles' instruction
// fetches competed, and a DCT32 selection row pass took about 7K cycles
// against 2.9K when its code was still cached. kOrdered is a separate
// instantiation so that the kernel without an order carries none of its
// index arithmetic (which slowed it by 0.6%).
template <bool kOrdered>
__global__ void __launch_bounds__(kPairThreads, 1)
    frontend_kernel(FrontendInputs in, FrontendScalars sc, FrontendTables tb, FrontendOutputs out) {
    extern __shared__ __align__(16) float smem[];
    const int half{static_cast<int>(threadIdx.x) / kThreads};
    int tx{2 * static_cast<int>(blockIdx.x) + half};
    int ty{static_cast<int>(blockIdx.y)};
    if constexpr (kOrdered) {
        // Entries 2b, 2b + 1 of the order for CTA b (raster over the grid,
        // which has at least ntiles / 2 CTAs).
        const int tiles_x{(in.width + kTile - 1) / kTile};
        const int ntiles{tiles_x * ((in.height + kTile - 1) / kTile)};
        const int slot{2 * (static_cast<int>(blockIdx.y * gridDim.x + blockIdx.x)) + half};
        if (slot >= ntiles) return;  // no barrier waits on it
        const int tile{static_cast<int>(in.tile_order[slot])};
        tx = tile % tiles_x;
        ty = tile / tiles_x;
    } else {
        if (tx * kTile >= in.width) return;  // the right half of an odd tile row: no barrier waits on it
    }
    frontend_tile(in, sc, tb, out, tx, ty, smem + half * (kTileSmemStride / sizeof(float)), 1 + half);
}

// One tile of a batched launch, kept out of line: inlined into the work loop,
// the tile's code held about 30 more registers live (its frame's fields and
// coordinates are run-time values here, where the single-frame kernel reads
// kernel parameters and block indices) and spilled 112 bytes per thread; out
// of line it needs no more registers than the single-frame kernel (8 x 4K
// batch: 1653 -> 1732 frames/s). The frame and tables are passed by value
// (read from the call's copy, not through a pointer into the parameter
// block): 1.8% fewer cycles per tile.
__device__ __noinline__ void batch_tile(const FrontendJob j, const FrontendTables tb, int local, float* smem,
                                       int bar) {
    frontend_tile(j.in, j.sc, tb, j.out, local % j.tiles_x, local / j.tiles_x, smem, bar);
}

// The frame of work-list item `item` and the item's tile within it.
__device__ __forceinline__ void batch_item(const FrontendBatch& b, std::uint32_t item, float* smem, int bar) {
    int f{0};
    while (f + 1 < b.nframes && b.jobs[f + 1].tile_begin <= item) ++f;
    const FrontendJob& j{b.jobs[f]};
    batch_tile(j, b.tb, static_cast<int>(item - j.tile_begin), smem, bar);
}

// Frames of a batch as one work list of tiles (frame j's tiles are items
// tile_begin .. tile_begin + tiles - 1): resident CTAs take items until the
// list is done, either claimed `chunk` at a time from a counter (dynamic) or
// every gridDim-th chunk (static). The claimed item travels through the
// Small::n32 word, which a tile writes before it reads it.
__global__ void __launch_bounds__(kThreads, 2) frontend_batch_kernel(const __grid_constant__ FrontendBatch b) {
    extern __shared__ __align__(16) float smem[];
    Small& sm{*reinterpret_cast<Small*>(smem + kRegionAFloats + 3 * kSplane)};
    const std::uint32_t chunk{static_cast<std::uint32_t>(b.chunk)};
    for (std::uint32_t round{0};; ++round) {
        std::uint32_t first;
        if (b.counter != nullptr) {
            if (threadIdx.x == 0) sm.n32 = static_cast<int>(atomicAdd(b.counter, chunk));
            __syncthreads();
            first = static_cast<std::uint32_t>(sm.n32);
            __syncthreads();
        } else {
            first = (round * gridDim.x + blockIdx.x) * chunk;
        }
        if (first >= b.total_tiles) break;
        const std::uint32_t last{min(first + chunk, b.total_tiles)};
        for (std::uint32_t item{first}; item < last; ++item) {
            batch_item(b, item, smem, 1);
            __syncthreads();
        }
    }
}

// The same work list taken two chunks at a time: half h of the CTA runs
// chunk h of each claim on its own tile memory and named barrier, so that,
// as in the single-frame kernel, two tiles run the same code together; both
// halves finish a claim before the next.
__global__ void __launch_bounds__(kPairThreads, 1)
    frontend_batch_pair_kernel(const __grid_constant__ FrontendBatch b) {
    extern __shared__ __align__(16) float smem[];
    const int half{static_cast<int>(threadIdx.x) / kThreads};
    float* tile_smem{smem + half * (kTileSmemStride / sizeof(float))};
    // The claim word is half 0's Small::n32; it is read before either tile
    // starts and written again only after both have finished.
    Small& sm{*reinterpret_cast<Small*>(smem + kRegionAFloats + 3 * kSplane)};
    const std::uint32_t chunk{static_cast<std::uint32_t>(b.chunk)};
    for (std::uint32_t round{0};; ++round) {
        std::uint32_t first;
        if (b.counter != nullptr) {
            if (threadIdx.x == 0) sm.n32 = static_cast<int>(atomicAdd(b.counter, 2 * chunk));
            __syncthreads();
            first = static_cast<std::uint32_t>(sm.n32);
            __syncthreads();
        } else {
            first = (round * gridDim.x + blockIdx.x) * 2 * chunk;
        }
        if (first >= b.total_tiles) break;
        const std::uint32_t mine{first + static_cast<std::uint32_t>(half) * chunk};
        const std::uint32_t last{min(mine + chunk, b.total_tiles)};
        for (std::uint32_t item{mine}; item < last; ++item) {
            batch_item(b, item, tile_smem, 1 + half);
            tile_sync(1 + half);
        }
        __syncthreads();
    }
}

}  // namespace

FrontendScalars frontend_scalars(float distance, std::uint32_t* global_scale,
                                 std::uint32_t* quant_dc) {
    // Quantiser calibration (src/quant_calibration.h:49-88).
    const float quant_ac{kAcQuant / distance};
    const float bt_dc{std::max(
        0.5f * distance,
        std::min(distance, kDcMul * std::pow((1.0f / kDcMul) * distance, kDcQuantPow)))};
    const float quant_dc_float{std::min(kDcQuant / bt_dc, 50.0f)};
    float scale{static_cast<float>(kGlobalScaleDenom) * quant_ac / kQuantFieldTarget};
    scale = scale < 1.0f ? 1.0f : scale;
    scale = scale > static_cast<float>(1 << 15) ? static_cast<float>(1 << 15) : scale;
    int gs{static_cast<int>(scale)};
    const int scaled_quant_dc{static_cast<int>(quant_dc_float * kGlobalScaleNumerator * 1.6f)};
    if (gs > scaled_quant_dc) {
        gs = scaled_quant_dc <= 0 ? 1 : scaled_quant_dc;
    }
    const float inv_gs{1.0f * static_cast<float>(kGlobalScaleDenom) / static_cast<float>(gs)};
    float fval{quant_dc_float * inv_gs + 0.5f};
    fval = std::min<float>(static_cast<float>(1 << 16), fval);
    const int qdc{static_cast<int>(fval)};
    int raw_q{static_cast<int>(std::lround(quant_ac * inv_gs))};
    raw_q = std::max(1, std::min(kQuantMax, raw_q));
    const float gsf{static_cast<float>(gs) * (1.0f / kGlobalScaleDenom)};

    FrontendScalars s{};
    // AQ mapping and FuzzyErosion weights (src/frontend_fused.cu:349-380).
    const float ascale{kAcQuant / distance};
    const float base_level{0.48f * ascale};
    float dampen{1.0f};
    if (distance >= 2.0f) {
        dampen = 1.0f - (distance - 2.0f) / (14.0f - 2.0f);
        if (dampen < 0.0f) {
            dampen = 0.0f;
        }
    }
    s.mul_pb = ascale * dampen;
    s.add_pb = (1.0f - dampen) * base_level;
    const float efm{distance < 2.0f ? (2.0f - distance) * 0.5f : 0.0f};
    float km0{0.125f};
    float km1{0.10f - efm * 0.10f};
    float km2{0.09f - efm * 0.09f};
    float km3{0.06f - efm * 0.06f};
    const float norm{0.29959705784054957f / (km0 + km1 + km2 + km3)};
    s.km0 = km0 * norm;
    s.km1 = km1 * norm;
    s.km2 = km2 * norm;
    s.km3 = km3 * norm;
    s.inv_global_scale = inv_gs;
    s.mask_sqrt_mul = std::sqrt(kMaskMul);
    s.qgsf_select = static_cast<float>(raw_q) * gsf;
    s.gsf = gsf;
    s.dc_scale = gsf * static_cast<float>(qdc);
    if (global_scale != nullptr) *global_scale = static_cast<std::uint32_t>(gs);
    if (quant_dc != nullptr) *quant_dc = static_cast<std::uint32_t>(qdc);
    return s;
}

bool frontend_tables_init(FrontendTables* tables) {
    // Bases.
    for (int n : {8, 16, 32}) {
        // Pair layout: element 2 * ((k / 2) * n + t) + (k & 1) holds basis[k][t].
        std::vector<float> sel(static_cast<std::size_t>(n) * n);
        std::vector<float> dct(static_cast<std::size_t>(n) * n);
        for (int k{0}; k < n; ++k) {
            const double g{k == 0 ? 1.0 / n : 1.4142135623730950488 / n};
            const float gf{k == 0 ? 1.0f / n : 1.4142135623730951f / n};
            for (int t{0}; t < n; ++t) {
                const int at{2 * ((k >> 1) * n + t) + (k & 1)};
                sel[at] = static_cast<float>(g * std::cos(3.14159265358979323846 * (t + 0.5) * k / n));
                const float arg{3.14159265358979323846f * (t + 0.5f) * k / n};
                dct[at] = gf * std::cos(arg);
            }
        }
        const void* sel_sym{n == 8 ? static_cast<const void*>(&c_sel8)
                                   : (n == 16 ? static_cast<const void*>(&c_sel16)
                                              : static_cast<const void*>(&c_sel32))};
        const void* dct_sym{n == 8 ? static_cast<const void*>(&c_dct8)
                                   : (n == 16 ? static_cast<const void*>(&c_dct16)
                                              : static_cast<const void*>(&c_dct32))};
        if (cudaMemcpyToSymbol(sel_sym, sel.data(), sel.size() * sizeof(float)) != cudaSuccess ||
            cudaMemcpyToSymbol(dct_sym, dct.data(), dct.size() * sizeof(float)) != cudaSuccess) {
            return false;
        }
    }
    // Dequantisation weights [size][channel][1024].
    std::vector<float> deq(3 * 3 * 1024, 0.0f);
    for (int c{0}; c < 3; ++c) {
        for (int i{0}; i < 64; ++i) std::memcpy(&deq[(0 * 3 + c) * 1024 + i], &kDequantBits8[c][i], 4);
        for (int i{0}; i < 256; ++i) std::memcpy(&deq[(1 * 3 + c) * 1024 + i], &kDequantBits16[c][i], 4);
        for (int i{0}; i < 1024; ++i) std::memcpy(&deq[(2 * 3 + c) * 1024 + i], &kDequantBits32[c][i], 4);
    }
    // Selection weights: DCT8 Y weight at (round(fx*8/N), round(fy*8/N)) clamped to 7.
    std::vector<float> sw(3 * 1024, 0.0f);
    for (int si{0}; si < 3; ++si) {
        const int n{8 << si};
        for (int fx{0}; fx < n; ++fx) {
            for (int fy{0}; fy < n; ++fy) {
                int sx{static_cast<int>(std::lround(fx * 8.0 / n))};
                int sy{static_cast<int>(std::lround(fy * 8.0 / n))};
                sx = sx > 7 ? 7 : sx;
                sy = sy > 7 ? 7 : sy;
                sw[si * 1024 + fx * n + fy] = deq[(0 * 3 + 1) * 1024 + sx * 8 + sy];
            }
        }
    }
    // log2f(1 + i) with the host libm: the rate proxy of the selection host twin.
    std::vector<float> l2(kLog2TableSize);
    for (int i{0}; i < kLog2TableSize; ++i) {
        l2[i] = std::log2(1.0f + static_cast<float>(i));
    }
    // Orthonormal m-point DCT basis for the LLF -> DC resampling, m = 2 and 4:
    // [m][k][n] stride 4 (src/vardct_layout.h:75-79).
    std::vector<double> ob(32, 0.0);
    for (int mi{0}; mi < 2; ++mi) {
        const int m{mi == 0 ? 2 : 4};
        const double md{static_cast<double>(m)};
        for (int k{0}; k < m; ++k) {
            for (int nn{0}; nn < m; ++nn) {
                const double normv{k == 0 ? std::sqrt(1.0 / md) : std::sqrt(2.0 / md)};
                ob[mi * 16 + k * 4 + nn] =
                    normv * std::cos(3.14159265358979323846 * (static_cast<double>(nn) + 0.5) *
                                     static_cast<double>(k) / md);
            }
        }
    }
    // Reciprocals RN(1 / w) after the weights (zero where an entry is unused).
    deq.resize(2 * deq.size());
    for (std::size_t i{0}; i < static_cast<std::size_t>(kDequantInv); ++i) {
        deq[kDequantInv + i] = deq[i] != 0.0f ? 1.0f / deq[i] : 0.0f;
    }
    float* d_deq{nullptr};
    float* d_sw{nullptr};
    float* d_l2{nullptr};
    double* d_ob{nullptr};
    if (cudaMalloc(&d_deq, deq.size() * 4) != cudaSuccess ||
        cudaMalloc(&d_sw, sw.size() * 4) != cudaSuccess ||
        cudaMalloc(&d_l2, l2.size() * 4) != cudaSuccess ||
        cudaMalloc(&d_ob, ob.size() * 8) != cudaSuccess) {
        return false;
    }
    if (cudaMemcpy(d_deq, deq.data(), deq.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_sw, sw.data(), sw.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_l2, l2.data(), l2.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_ob, ob.data(), ob.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess) {
        return false;
    }
    tables->dequant = d_deq;
    tables->sel_weight = d_sw;
    tables->log2_1p = d_l2;
    tables->llf_basis = d_ob;
    return cudaFuncSetAttribute(frontend_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(2 * kTileSmemStride)) == cudaSuccess &&
           cudaFuncSetAttribute(frontend_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(2 * kTileSmemStride)) == cudaSuccess &&
           cudaFuncSetAttribute(frontend_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(kSmemBytes)) == cudaSuccess &&
           cudaFuncSetAttribute(frontend_batch_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(2 * kTileSmemStride)) == cudaSuccess;
}

bool frontend_launch(const FrontendInputs& in, const FrontendScalars& s, const FrontendTables& t,
                     const FrontendOutputs& out, void* stream) {
    const int tiles_x{(in.width + kTile - 1) / kTile};
    const dim3 grid{static_cast<unsigned>((tiles_x + 1) / 2), static_cast<unsigned>((in.height + kTile - 1) / kTile)};
    if (in.tile_order != nullptr) {
        frontend_kernel<true><<<grid, kPairThreads, 2 * kTileSmemStride, static_cast<cudaStream_t>(stream)>>>(in, s, t,
                                                                                                           out);
    } else {
        frontend_kernel<false><<<grid, kPairThreads, 2 * kTileSmemStride, static_cast<cudaStream_t>(stream)>>>(in, s, t,
                                                                                                            out);
    }
    return cudaGetLastError() == cudaSuccess;
}

bool frontend_batch_launch(const FrontendBatch& b, int ctas, bool paired, void* stream) {
    if (b.nframes <= 0 || b.nframes > kBatchFrames || ctas <= 0 || b.chunk <= 0) return false;
    cudaStream_t st{static_cast<cudaStream_t>(stream)};
    if (paired) {
        frontend_batch_pair_kernel<<<static_cast<unsigned>(ctas), kPairThreads, 2 * kTileSmemStride, st>>>(b);
    } else {
        frontend_batch_kernel<<<static_cast<unsigned>(ctas), kThreads, kSmemBytes, st>>>(b);
    }
    return cudaGetLastError() == cudaSuccess;
}

}  // namespace jxb
