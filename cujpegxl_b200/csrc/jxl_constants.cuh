// Numeric constants of the encode path and small integer helpers shared by the
// host orchestration and the kernels.
//
// The values are format or encoder constants that must equal the reference
// encoder's bit for bit (the test suite compares them with the reference
// checker library): libjxl's opsin absorbance matrix and bias, BT.709 full
// range Y'CbCr -> R'G'B', inverse-gaborish weights, adaptive-quantisation
// constants, quantiser calibration constants, chroma-from-luma factors and the
// default VarDCT AC context model. Each block cites where the reference
// defines the same quantity.
#pragma once

#include <cstddef>
#include <cstdint>

#include "jxl_math.cuh"

namespace jxb {

// ---- geometry -----------------------------------------------------------------
constexpr int kBlock = 8;                  // 8x8 DCT block
constexpr int kRegionBlocks = 4;           // 32x32 transform-selection region
constexpr int kTileBlocks = 8;             // 64x64 chroma-from-luma colour tile
constexpr int kAcGroupBlocks = 32;         // 256x256 AC group
constexpr int kDcGroupBlocks = 256;        // 2048x2048 DC group
constexpr int kCoeffsPerBlock = 64;        // covered-block slots per 8x8 position
constexpr int kHistStride = 256;           // token alphabet bound per histogram
constexpr int kNumClusters = 32;           // fixed AC cluster count
constexpr std::int8_t kAcsCovered = 0;     // acs value of a covered 8x8 block

// ---- colour (reference src/xyb_impl.cuh:17-35) -----------------------------------
constexpr float kM00 = 0.30f;
constexpr float kM02 = 0.078f;
constexpr float kM01 = 1.0f - kM02 - kM00;
constexpr float kM10 = 0.23f;
constexpr float kM12 = 0.078f;
constexpr float kM11 = 1.0f - kM12 - kM10;
constexpr float kM20 = 0.24342268924547819f;
constexpr float kM21 = 0.20476744424496821f;
constexpr float kM22 = 1.0f - kM20 - kM21;
constexpr float kOpsinBias = 0.0037930732552754493f;
// -cbrt(kOpsinBias), rounded from double.
constexpr float kNegCbrtBias = -0.15595419704914093f;
constexpr float kCrToR = 1.5748f;
constexpr float kCbToG = 0.1873242729f;
constexpr float kCrToG = 0.4681242729f;
constexpr float kCbToB = 1.8556f;
constexpr float kChromaCenter = 128.0f / 255.0f;
constexpr float kInv255 = 1.0f / 255.0f;

// ---- inverse gaborish (reference src/gaborish.h:16-28) ---------------------------
constexpr float kGabK0 = -0.09495815671340026f;
constexpr float kGabK1 = -0.041031725066768575f;
constexpr float kGabK2 = 0.013710004822696948f;
constexpr float kGabK3 = 0.006510206083837737f;
constexpr float kGabK4 = -0.0014789063378272242f;
constexpr float kGabNorm = 1.0f / (1.0f + 4.0f * (kGabK0 + kGabK1 + kGabK2 + kGabK4 + 2.0f * kGabK3));
constexpr float kGabC = kGabNorm;             // centre
constexpr float kGabEdge = kGabNorm * kGabK0; // (+-1, 0), (0, +-1)
constexpr float kGabEdge2 = kGabNorm * kGabK2;// (+-2, 0), (0, +-2)
constexpr float kGabDiag = kGabNorm * kGabK1; // (+-1, +-1)
constexpr float kGabKnight = kGabNorm * kGabK3;  // (+-2, +-1), (+-1, +-2)
constexpr float kGabDiag2 = kGabNorm * kGabK4;   // (+-2, +-2)

// ---- adaptive quantisation (reference src/adaptive_quant_impl.cuh:16-27,44-76,
//      src/frontend_fused.cu:139-196) --------------------------------------------
constexpr float kMatchGammaOffset = 0.019f;
constexpr float kDiffLimit = 0.2f;
constexpr float kSgMul = 226.77216153508914f;
constexpr float kSgMul2 = 1.0f / 73.377132366608819f;
constexpr float kSgLog2 = 0.693147181f;
constexpr float kSgRetMul = kSgMul2 * 18.6580932135f * kSgLog2;
constexpr float kSgVOffset = 7.7825991679894591f;
constexpr float kRatioEps = 1e-2f;
constexpr float kRatioNumMul = kSgRetMul * 3.0f * kSgMul;
constexpr float kRatioVOffset = kSgVOffset * kSgLog2 + kRatioEps;
constexpr float kRatioDenMul = kSgLog2 * kSgMul;
constexpr float kMaskLogOffset = 27.505837037000106f;
constexpr float kMaskMul = 211.66567973503678f * 1e8f;
constexpr float kMaskBase = -0.7647f;
constexpr float kMaskMul4 = 9.4708735624378946f;
constexpr float kMaskMul2 = 17.35036561631863f;
constexpr float kMaskOffset2 = 302.59587815579727f;
constexpr float kMaskMul3 = 6.7943250517376494f;
constexpr float kMaskOffset3 = 3.7179635626140772f;
constexpr float kMaskOffset4 = 0.25f * kMaskOffset3;
constexpr float kMaskMul0 = 0.80061762862741759f;
constexpr float kHfValMin = 0.0206f;
constexpr float kGammaBias = 0.16f;
constexpr float kBlueLimit = 0.027121074570634722f;
constexpr float kBlueOffset = 0.084381641171960495f;
constexpr float kBlueMaxLimit = 15.398788439047934f;
constexpr float kHfMul = -0.38f;
constexpr float kHfAdd = 0.42f;
constexpr float kGammaLogMul = 0.1005613337192697f;
constexpr float kBlueMul = 0.14207000358439159f;

// ---- quantiser calibration (reference src/quant_calibration.h:16-34) ---------------
constexpr float kDcInvQuant[3] = {4096.0f, 512.0f, 256.0f};
constexpr float kAcQuant = 0.725f;
constexpr float kDcQuant = 1.095924047623553f;
constexpr float kDcQuantPow = 0.83f;
constexpr float kDcMul = 0.3f;
constexpr float kQuantFieldTarget = 5.0f;
constexpr int kGlobalScaleDenom = 1 << 16;
constexpr int kGlobalScaleNumerator = 4096;
constexpr int kQuantMax = 256;

// ---- transform selection (reference src/transform_select_impl.cuh:19-31) ---------
constexpr float kSelectLambda = 6.0e-4f;
constexpr float kSelectSplitEps = 1.0e-6f;
constexpr int kSelectPartials = 256;

// ---- chroma from luma (reference src/cfl.h:26-33) -------------------------------
constexpr int kCflColorFactor = 84;
constexpr float kCflColorScale = 1.0f / kCflColorFactor;
constexpr float kCflBaseB = 1.0f;

// ---- AC context model (libjxl default BlockCtxMap; reference src/ac_context.h) ---
constexpr int kNumBlockCtx = 15;
constexpr int kNonZeroBuckets = 37;
constexpr int kZeroDensityCount = 458;
constexpr int kNumAcContexts = kNumBlockCtx * (kNonZeroBuckets + kZeroDensityCount);  // 7425

// Block context of physical channel c (0=X, 1=Y, 2=B) for transform side n.
// Only the three square strategies are emitted: DCT8 (order 0), DCT16 (order
// 2) and DCT32 (order 3); the default map gives Y {0,2,2} and X/B {7,9,9}.
JX_HD int block_ctx(int c, int n) {
    const int ord_ctx{n == 8 ? 0 : 2};
    return c == 1 ? ord_ctx : 7 + ord_ctx;
}

// libjxl kCoeffFreqContext[k] for k in [1, 63].
JX_HD std::uint32_t coeff_freq_ctx(std::uint32_t k) {
    if (k < 16) return k - 1;
    if (k < 32) return 15 + (k - 16) / 2;
    return 23 + (k - 32) / 4;
}

// libjxl kCoeffNumNonzeroContext[nz] for nz in [1, 63].
JX_HD std::uint32_t coeff_nz_ctx(std::uint32_t nz) {
    if (nz < 2) return 0;
    if (nz < 3) return 31;
    if (nz < 5) return 62;
    if (nz < 9) return 93;
    if (nz < 13) return 123;
    if (nz < 21) return 152;
    if (nz < 33) return 180;
    return 206;
}

// Context of the non-zero-count token (libjxl NonZeroContext).
JX_HD std::uint32_t nonzero_context(std::uint32_t predicted, int bctx) {
    const std::uint32_t nz{predicted >= 64 ? 64u : predicted};
    const std::uint32_t c{nz < 8 ? nz : 4 + nz / 2};
    return c * kNumBlockCtx + static_cast<std::uint32_t>(bctx);
}

// Context of a coefficient token (libjxl ZeroDensityContext + block offset).
JX_HD std::uint32_t coeff_context(int bctx, std::uint32_t nz_left, std::uint32_t k,
                                  std::uint32_t covered, std::uint32_t log2_covered,
                                  std::uint32_t prev) {
    const std::uint32_t left{(nz_left + covered - 1) >> log2_covered};
    const std::uint32_t kk{k >> log2_covered};
    return static_cast<std::uint32_t>(kNumBlockCtx * kNonZeroBuckets + kZeroDensityCount * bctx) +
           (coeff_nz_ctx(left) + coeff_freq_ctx(kk)) * 2 + prev;
}

// Fixed 7425 -> 32 cluster map: luma/chroma split, then 4 non-zero-count bands
// and 12 zero-density bands (reference src/ac_context.h:101-129).
JX_HD int context_cluster(std::uint32_t ctx) {
    constexpr std::uint32_t kCount{kNumBlockCtx * kNonZeroBuckets};
    if (ctx < kCount) {
        const std::uint32_t bucket{ctx / kNumBlockCtx};
        const int group{static_cast<int>(ctx % kNumBlockCtx) < 7 ? 0 : 1};
        const int band{bucket < 4 ? 0 : (bucket < 12 ? 1 : (bucket < 24 ? 2 : 3))};
        return group * 4 + band;
    }
    const std::uint32_t rel{ctx - kCount};
    const int group{static_cast<int>(rel / kZeroDensityCount) < 7 ? 0 : 1};
    const std::uint32_t z{rel % kZeroDensityCount};
    int band;
    if (z < 160) {
        band = static_cast<int>(z / 32);
    } else if (z < 280) {
        band = 5 + static_cast<int>((z - 160) / 40);
    } else {
        band = z < 424 ? 8 + static_cast<int>((z - 280) / 48) : 11;
    }
    return 8 + group * 12 + band;
}

// libjxl PredictFromTopAndLeft on the group-local normalised non-zero grid.
JX_HD std::uint32_t predict_nonzeros(bool has_left, bool has_top, std::uint32_t top,
                                     std::uint32_t left) {
    if (!has_left) return has_top ? top : 32u;
    if (!has_top) return left;
    return (top + left + 1) / 2;
}

// libjxl ClampedGradient on (left, top, topleft) with modular edge rules.
JX_HD std::int32_t gradient_predict(bool has_left, bool has_top, std::int32_t w, std::int32_t n,
                                    std::int32_t nw) {
    const std::int32_t left{has_left ? w : (has_top ? n : 0)};
    const std::int32_t top{has_top ? n : left};
    const std::int32_t tl{(has_left && has_top) ? nw : left};
    const std::int32_t lo{left < top ? left : top};
    const std::int32_t hi{left < top ? top : left};
    if (tl < lo) return hi;
    if (tl > hi) return lo;
    return static_cast<std::int32_t>(static_cast<std::int64_t>(left) + top - tl);
}

// Hybrid-uint (4, 2, 0) split of a value into token, extra-bit count and bits.
JX_HD void hybrid_uint(std::uint32_t v, std::uint32_t& tok, std::uint32_t& nbits,
                       std::uint32_t& bits) {
    if (v < 16u) {
        tok = v;
        nbits = 0;
        bits = 0;
        return;
    }
#if defined(__CUDA_ARCH__)
    const std::uint32_t n{31u - static_cast<std::uint32_t>(__clz(v))};
#else
    const std::uint32_t n{31u - static_cast<std::uint32_t>(__builtin_clz(v))};
#endif
    const std::uint32_t m{v - (1u << n)};
    tok = 16u + ((n - 4u) << 2) + (m >> (n - 2u));
    nbits = n - 2u;
    bits = v & ((1u << nbits) - 1u);
}

JX_HD std::uint32_t pack_signed(std::int32_t v) {
    return (static_cast<std::uint32_t>(v) << 1) ^ static_cast<std::uint32_t>(v >> 31);
}

// libjxl AcStrategy raw type for the emitted sides: DCT 0, DCT16X16 4, DCT32X32 5.
JX_HD std::int32_t raw_strategy(int side) { return side == 16 ? 4 : (side == 32 ? 5 : 0); }

// Covered-block slot of raw coefficient r of a side-n first-block at (bx, by):
// covered ordinal q = r / 64 selects block (by + q / (n/8), bx + q % (n/8)),
// r % 64 is the slot (reference src/vardct_layout.h:54-62).
JX_HD std::size_t covered_slot(int n, std::size_t bx, std::size_t by, std::size_t bw, int r) {
    const int side{n / 8};
    const int q{r >> 6};
    return ((by + static_cast<std::size_t>(q / side)) * bw + bx + static_cast<std::size_t>(q % side)) *
               kCoeffsPerBlock +
           static_cast<std::size_t>(r & 63);
}

}  // namespace jxb
