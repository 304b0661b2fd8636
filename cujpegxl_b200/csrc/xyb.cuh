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

// ---- Two pixels per thread on the packed f32x2 instructions ----------------
// Each component of __fmul2_rn / __fadd2_rn / __ffma2_rn rounds exactly as the
// scalar instruction, so every function below returns, per component, the bits
// of its scalar counterpart above (x - c is computed as x + (-c), which is the
// same IEEE operation).

__device__ __forceinline__ float2 f2dup(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 f2neg(float2 v) { return make_float2(-v.x, -v.y); }

// The factors jx_pow24 derives from the exponent, for x in [2^-5, 2), by
// exponent byte e - 122 (e in 122..127, k = e - 127 in [-5, 0]):
// {c = 2^(0.4 r), 2^(2 floor(k / 5))} with r = k - 5 floor(k / 5).
__host__ __device__ constexpr float pow24_factor_c(int i) {
    return i == 1 ? 1.31950791077289425f
                  : (i == 2 ? 1.74110112659224828f
                            : (i == 3 ? 2.29739670999407037f : (i == 4 ? 3.03143313302079624f : 1.0f)));
}
__host__ __device__ constexpr float pow24_factor_scale(int i) { return i == 5 ? 1.0f : 0.25f; }

// jx_pow24 on both components, for x in [2^-5, 2); lut[i] = {pow24_factor_c(i), pow24_factor_scale(i)}
// (a shared-memory copy: one 8-byte load per component replaces the
// exponent arithmetic). The sRGB transfer only calls it on (e + 0.055) / 1.055
// with e in [0, 1], which lies in [0.052, 1.0000002].
__device__ __forceinline__ float2 jx_pow24_2(float2 x, const float2* lut) {
    float2 m, c, scale;
    {
        const std::uint32_t u[2]{f2u(x.x), f2u(x.y)};
        float mm[2], cc[2], ss[2];
#pragma unroll
        for (int h{0}; h < 2; ++h) {
            mm[h] = u2f((u[h] & 0x7fffffu) | 0x3f800000u);
            const float2 f{lut[static_cast<int>(u[h] >> 23) - 122]};
            cc[h] = f.x;
            ss[h] = f.y;
        }
        m = make_float2(mm[0], mm[1]);
        c = make_float2(cc[0], cc[1]);
        scale = make_float2(ss[0], ss[1]);
    }
    const float2 v{__fadd2_rn(m, f2dup(-1.5f))};
    float2 p{__ffma2_rn(f2dup(-8.58357804e-04f), v, f2dup(1.51637842e-03f))};
    p = __ffma2_rn(p, v, f2dup(-2.33355959e-03f));
    p = __ffma2_rn(p, v, f2dup(4.58948039e-03f));
    p = __ffma2_rn(p, v, f2dup(-9.66759456e-03f));
    p = __ffma2_rn(p, v, f2dup(2.23054436e-02f));
    p = __ffma2_rn(p, v, f2dup(-6.27241061e-02f));
    p = __ffma2_rn(p, v, f2dup(3.13621006e-01f));
    p = __ffma2_rn(p, v, f2dup(1.17607902e+00f));
    return __fmul2_rn(__fmul2_rn(__fmul2_rn(x, x), __fmul2_rn(p, c)), scale);
}

// jx_cbrt on both components.
__device__ __forceinline__ float2 jx_cbrt2(float2 x) {
    float2 r{u2f(0x54a2fa8cu - f2u(x.x) / 3u), u2f(0x54a2fa8cu - f2u(x.y) / 3u)};
    const float2 nx{f2neg(x)};
    const float2 third{f2dup(0.333333343f)};
#pragma unroll
    for (int it{0}; it < 3; ++it) {
        const float2 t{__fmul2_rn(__fmul2_rn(r, r), r)};
        const float2 e{__ffma2_rn(nx, t, f2dup(1.0f))};
        r = __ffma2_rn(__fmul2_rn(r, third), e, r);
    }
    float2 y{__fmul2_rn(__fmul2_rn(x, r), r)};
    const float2 y2{__fmul2_rn(y, y)};
    const float2 res{__ffma2_rn(y2, y, nx)};
    y = __ffma2_rn(f2neg(res), __fmul2_rn(__fmul2_rn(r, r), third), y);
    return y;
}

__device__ __forceinline__ float2 clamp01_2(float2 v) { return make_float2(clamp01(v.x), clamp01(v.y)); }

// srgb_to_linear on both components (both branches evaluated, one kept),
// for e in [0, 1].
__device__ __forceinline__ float2 srgb_to_linear2(float2 e, const float2* lut) {
    const float2 lin{__fmul2_rn(e, f2dup(1.0f / 12.92f))};
    const float2 pw{jx_pow24_2(__fmul2_rn(__fadd2_rn(e, f2dup(0.055f)), f2dup(1.0f / 1.055f)), lut)};
    return make_float2(e.x <= 0.04045f ? lin.x : pw.x, e.y <= 0.04045f ? lin.y : pw.y);
}

// Cb/Cr tap sums of pixel column gx on chroma rows (ya, yb) with weights
// (wya, wyb), as in xyb_pixel.
template <int kWin>
__device__ __forceinline__ void chroma_taps(const std::uint8_t* win, int cx0, int cy0, int gx, int cw, int ya,
                                            int yb, int wya, int wyb, int& scb, int& scr) {
    const int jx{gx >> 1};
    int xa, xb, wxa, wxb;
    if (gx & 1) {
        xa = jx; xb = min(jx + 1, cw - 1); wxa = 3; wxb = 1;
    } else {
        xa = max(jx - 1, 0); xb = jx; wxa = 1; wxb = 3;
    }
    const int aa{2 * ((ya - cy0) * kWin + xa - cx0)};
    const int ab{2 * ((ya - cy0) * kWin + xb - cx0)};
    const int ba{2 * ((yb - cy0) * kWin + xa - cx0)};
    const int bb{2 * ((yb - cy0) * kWin + xb - cx0)};
    scb = wya * (wxa * win[aa] + wxb * win[ab]) + wyb * (wxa * win[ba] + wxb * win[bb]);
    scr = wya * (wxa * win[aa + 1] + wxb * win[ab + 1]) + wyb * (wxa * win[ba + 1] + wxb * win[bb + 1]);
}

// div4080 on both components.
__device__ __forceinline__ float2 div4080_2(int s0, int s1) {
    constexpr float kInv{1.0f / 4080.0f};
    const float2 sf{static_cast<float>(s0), static_cast<float>(s1)};
    const float2 q0{__fmul2_rn(sf, f2dup(kInv))};
    return __ffma2_rn(__ffma2_rn(f2neg(q0), f2dup(4080.0f), sf), f2dup(kInv), q0);
}

// xyb_pixel for pixels (gx0, gy) and (gx1, gy) of one row: component 0 of
// each output is the first pixel, component 1 the second. lut: the factor
// table of jx_pow24_2. The window's (cb, cr) pairs start at even
// byte offsets.
template <int kWin>
__device__ __forceinline__ void xyb_pixel2(int luma0, int luma1, const std::uint8_t* win, int cx0, int cy0, int gx0,
                                           int gx1, int gy, int width, int height, const float2* lut, float2& ox,
                                           float2& oy, float2& ob) {
    const float2 yv{__fmul2_rn(make_float2(static_cast<float>(luma0), static_cast<float>(luma1)), f2dup(kInv255))};
    const int cw{width >> 1};
    const int ch{height >> 1};
    const int jy{gy >> 1};
    int ya, yb, wya, wyb;
    if (gy & 1) {
        ya = jy; yb = min(jy + 1, ch - 1); wya = 3; wyb = 1;
    } else {
        ya = max(jy - 1, 0); yb = jy; wya = 1; wyb = 3;
    }
    int scb0, scr0, scb1, scr1;
    if ((gx0 & 1) == 0 && gx1 == gx0 + 1) {
        // An even pixel and its right neighbour share chroma column jx: the
        // even one takes columns (jx - 1, jx) with weights (1, 3), the odd
        // one (jx, jx + 1) with (3, 1), clamped as in chroma_taps. Three
        // 16-bit (cb, cr) loads per chroma row.
        const int jx{gx0 >> 1};
        const int k0{max(jx - 1, 0) - cx0};
        const int k1{jx - cx0};
        const int k2{min(jx + 1, cw - 1) - cx0};
        const auto* ra{reinterpret_cast<const std::uint16_t*>(win) + (ya - cy0) * kWin};
        const auto* rb{reinterpret_cast<const std::uint16_t*>(win) + (yb - cy0) * kWin};
        const int a0{ra[k0]}, a1{ra[k1]}, a2{ra[k2]};
        const int b0{rb[k0]}, b1{rb[k1]}, b2{rb[k2]};
        scb0 = wya * ((a0 & 0xff) + 3 * (a1 & 0xff)) + wyb * ((b0 & 0xff) + 3 * (b1 & 0xff));
        scr0 = wya * ((a0 >> 8) + 3 * (a1 >> 8)) + wyb * ((b0 >> 8) + 3 * (b1 >> 8));
        scb1 = wya * (3 * (a1 & 0xff) + (a2 & 0xff)) + wyb * (3 * (b1 & 0xff) + (b2 & 0xff));
        scr1 = wya * (3 * (a1 >> 8) + (a2 >> 8)) + wyb * (3 * (b1 >> 8) + (b2 >> 8));
    } else {
        chroma_taps<kWin>(win, cx0, cy0, gx0, cw, ya, yb, wya, wyb, scb0, scr0);
        chroma_taps<kWin>(win, cx0, cy0, gx1, cw, ya, yb, wya, wyb, scb1, scr1);
    }
    const float2 cb{__fadd2_rn(div4080_2(scb0, scb1), f2dup(-kChromaCenter))};
    const float2 cr{__fadd2_rn(div4080_2(scr0, scr1), f2dup(-kChromaCenter))};

    const float2 r{clamp01_2(srgb_to_linear2(clamp01_2(__ffma2_rn(f2dup(kCrToR), cr, yv)), lut))};
    const float2 g{clamp01_2(srgb_to_linear2(
        clamp01_2(__ffma2_rn(f2dup(-kCrToG), cr, __ffma2_rn(f2dup(-kCbToG), cb, yv))), lut))};
    const float2 b{clamp01_2(srgb_to_linear2(clamp01_2(__ffma2_rn(f2dup(kCbToB), cb, yv)), lut))};

    const float2 bias{f2dup(kOpsinBias)};
    float2 m0{__fadd2_rn(__ffma2_rn(f2dup(kM02), b, __ffma2_rn(f2dup(kM01), g, __fmul2_rn(f2dup(kM00), r))), bias)};
    float2 m1{__fadd2_rn(__ffma2_rn(f2dup(kM12), b, __ffma2_rn(f2dup(kM11), g, __fmul2_rn(f2dup(kM10), r))), bias)};
    float2 m2{__fadd2_rn(__ffma2_rn(f2dup(kM22), b, __ffma2_rn(f2dup(kM21), g, __fmul2_rn(f2dup(kM20), r))), bias)};
    const float2 nb{f2dup(kNegCbrtBias)};
    m0 = __fadd2_rn(jx_cbrt2(make_float2(fmaxf(m0.x, 0.0f), fmaxf(m0.y, 0.0f))), nb);
    m1 = __fadd2_rn(jx_cbrt2(make_float2(fmaxf(m1.x, 0.0f), fmaxf(m1.y, 0.0f))), nb);
    m2 = __fadd2_rn(jx_cbrt2(make_float2(fmaxf(m2.x, 0.0f), fmaxf(m2.y, 0.0f))), nb);
    ox = __fmul2_rn(f2dup(0.5f), __fadd2_rn(m0, f2neg(m1)));
    oy = __fmul2_rn(f2dup(0.5f), __fadd2_rn(m0, m1));
    ob = m2;
}

}  // namespace jxb
