// NV12 -> XYB pixel conversion shared by the fused frontend and the
// transform-decision network's inference kernel, so that both see the same
// XYB values bit for bit. Compiled with -fmad=false like every file here.
#pragma once

#include <cstdint>

#include "jxl_constants.cuh"
#include "jxl_math.cuh"

namespace jxb {

__device__ __forceinline__ float clamp01(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

// sRGB transfer function to linear (src/xyb_impl.cuh:37-40).
__device__ __forceinline__ float srgb_to_linear(float e) {
    return e <= 0.04045f ? e * (1.0f / 12.92f) : jx_pow24((e + 0.055f) * (1.0f / 1.055f));
}

// s / 4080.0f correctly rounded for an integer s in [0, 4080], without a
// division: q0 = s * RN(1/4080), then one Newton correction with the exact
// residual s - q0 * 4080. Checked against the rounded quotient for every s in
// the range (the tap sums of the chroma upsample never leave it).
__device__ __forceinline__ float div4080(int s) {
    constexpr float kInv{1.0f / 4080.0f};
    const float sf{static_cast<float>(s)};
    const float q0{sf * kInv};
    return jx_fma(jx_fma(-q0, 4080.0f, sf), kInv, q0);
}

// NV12 pixel (gx, gy) -> XYB (src/xyb_impl.cuh:49-70), from its luma byte and
// a chroma window of kWin x kWin (cb, cr) pairs in shared memory whose first
// pair is chroma sample (cx0, cy0). Chroma is the centred bilinear 2x upsample
// of the texture path (src/frontend_fused.cu:222), taken exactly: the four
// taps carry weights {1,3}x{1,3}/16, summed in integers.
template <int kWin>
__device__ __forceinline__ void xyb_pixel(int luma, const std::uint8_t* win, int cx0, int cy0, int gx, int gy,
                                          int width, int height, float& ox, float& oy, float& ob) {
    const float yv{static_cast<float>(luma) * kInv255};
    const int cw{width >> 1};
    const int ch{height >> 1};
    const int jx{gx >> 1};
    const int jy{gy >> 1};
    int xa, xb, wxa, wxb, ya, yb, wya, wyb;
    if (gx & 1) {
        xa = jx; xb = min(jx + 1, cw - 1); wxa = 3; wxb = 1;
    } else {
        xa = max(jx - 1, 0); xb = jx; wxa = 1; wxb = 3;
    }
    if (gy & 1) {
        ya = jy; yb = min(jy + 1, ch - 1); wya = 3; wyb = 1;
    } else {
        ya = max(jy - 1, 0); yb = jy; wya = 1; wyb = 3;
    }
    const int aa{2 * ((ya - cy0) * kWin + xa - cx0)};
    const int ab{2 * ((ya - cy0) * kWin + xb - cx0)};
    const int ba{2 * ((yb - cy0) * kWin + xa - cx0)};
    const int bb{2 * ((yb - cy0) * kWin + xb - cx0)};
    const int scb{wya * (wxa * win[aa] + wxb * win[ab]) + wyb * (wxa * win[ba] + wxb * win[bb])};
    const int scr{wya * (wxa * win[aa + 1] + wxb * win[ab + 1]) + wyb * (wxa * win[ba + 1] + wxb * win[bb + 1])};
    const float cb{div4080(scb) - kChromaCenter};
    const float cr{div4080(scr) - kChromaCenter};

    const float r{clamp01(srgb_to_linear(clamp01(jx_fma(kCrToR, cr, yv))))};
    const float g{clamp01(srgb_to_linear(clamp01(jx_fma(-kCrToG, cr, jx_fma(-kCbToG, cb, yv)))))};
    const float b{clamp01(srgb_to_linear(clamp01(jx_fma(kCbToB, cb, yv))))};

    float m0{jx_fma(kM02, b, jx_fma(kM01, g, kM00 * r)) + kOpsinBias};
    float m1{jx_fma(kM12, b, jx_fma(kM11, g, kM10 * r)) + kOpsinBias};
    float m2{jx_fma(kM22, b, jx_fma(kM21, g, kM20 * r)) + kOpsinBias};
    m0 = jx_cbrt(fmaxf(m0, 0.0f)) + kNegCbrtBias;
    m1 = jx_cbrt(fmaxf(m1, 0.0f)) + kNegCbrtBias;
    m2 = jx_cbrt(fmaxf(m2, 0.0f)) + kNegCbrtBias;
    ox = 0.5f * (m0 - m1);
    oy = 0.5f * (m0 + m1);
    ob = m2;
}

}  // namespace jxb
