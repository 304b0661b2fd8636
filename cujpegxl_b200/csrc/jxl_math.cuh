// Deterministic single-precision math for the encoder's float stages.
//
// Every function here is built only from IEEE-754 single operations that are
// correctly rounded on both the GPU and the host (add, sub, mul, div, fmaf,
// rint, exponent bit manipulation), so the same inputs give the same bits on
// the B200 and in a CPU restatement compiled without contraction. This matters
// because integer decisions downstream (adaptive quant field, quantised
// coefficients) are taken from these floats and must agree bit for bit.
//
// Methods (all written from the mathematics, not from any library's code):
//  - log2: argument reduction m*2^e with m in (sqrt(1/2), sqrt(2)], then the
//    atanh series log(m) = 2 artanh(s), s = (m-1)/(m+1), to s^9.
//  - exp2: n = rint(y), f = y - n in [-1/2, 1/2], Taylor series of e^(f ln 2)
//    to degree 8, then an exact scaling by 2^n through the exponent bits.
//  - exp: Cody-Waite reduction x - n*ln2 (two-term ln2) and the Taylor series
//    of e^r to degree 8.
//  - cbrt: bit-level seed for x^(-1/3), four Newton steps on the inverse cube
//    root (division free), then one correction step on the cube root itself.
//  - pow(x, 2.4) = x^2 * 2^(0.4 log2 x), keeping the exponent small so the
//    absolute error of the exponent stays near one float ulp.
// Accuracy (checked by the test suite against double precision): a few ulp,
// far inside the 1e-5 relative tolerance the float stages are held to.
#pragma once

#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define JX_HD __host__ __device__ __forceinline__
#else
#define JX_HD inline
#endif

namespace jxb {

JX_HD std::uint32_t f2u(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    std::uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
#endif
}

JX_HD float u2f(std::uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    std::memcpy(&f, &u, 4);
    return f;
#endif
}

JX_HD float jx_fma(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return __builtin_fmaf(a, b, c);
#endif
}

JX_HD float jx_rint(float x) {
#if defined(__CUDA_ARCH__)
    return rintf(x);
#else
    return __builtin_rintf(x);
#endif
}

// log2 for positive normal x.
JX_HD float jx_log2(float x) {
    const std::uint32_t u{f2u(x)};
    int e{static_cast<int>((u >> 23) & 0xffu) - 127};
    float m{u2f((u & 0x7fffffu) | 0x3f800000u)};
    if (m > 1.41421356f) {
        m = m * 0.5f;
        e += 1;
    }
    const float s{(m - 1.0f) / (m + 1.0f)};
    const float s2{s * s};
    float p{0.32059889797532520f};          // 2/(9 ln 2)
    p = jx_fma(p, s2, 0.41219858311113244f);  // 2/(7 ln 2)
    p = jx_fma(p, s2, 0.57707801635558536f);  // 2/(5 ln 2)
    p = jx_fma(p, s2, 0.96179669392597560f);  // 2/(3 ln 2)
    p = jx_fma(p, s2, 2.88539008177792681f);  // 2/ln 2
    return static_cast<float>(e) + s * p;
}

// 2^y for |y| < 120.
JX_HD float jx_exp2(float y) {
    const float n{jx_rint(y)};
    const float f{y - n};
    float p{1.3215486790144307e-06f};        // ln2^8/8!
    p = jx_fma(p, f, 1.5252733804059840e-05f);  // ln2^7/7!
    p = jx_fma(p, f, 1.5403530393381609e-04f);  // ln2^6/6!
    p = jx_fma(p, f, 1.3333558146428443e-03f);  // ln2^5/5!
    p = jx_fma(p, f, 9.6181291076284772e-03f);  // ln2^4/4!
    p = jx_fma(p, f, 5.5504108664821580e-02f);  // ln2^3/3!
    p = jx_fma(p, f, 2.4022650695910071e-01f);  // ln2^2/2!
    p = jx_fma(p, f, 6.9314718055994531e-01f);  // ln2
    p = jx_fma(p, f, 1.0f);
    const int ni{static_cast<int>(n)};
    return p * u2f(static_cast<std::uint32_t>(ni + 127) << 23);
}

// e^x for |x| < 80.
JX_HD float jx_exp(float x) {
    const float n{jx_rint(x * 1.44269504088896341f)};
    float r{jx_fma(-n, 0.693145751953125f, x)};      // ln2 high part (exact in 16 bits)
    r = jx_fma(-n, 1.42860682030941723e-06f, r);     // ln2 - high part
    float p{2.4801587301587302e-05f};                // 1/8!
    p = jx_fma(p, r, 1.9841269841269841e-04f);       // 1/7!
    p = jx_fma(p, r, 1.3888888888888889e-03f);       // 1/6!
    p = jx_fma(p, r, 8.3333333333333333e-03f);       // 1/5!
    p = jx_fma(p, r, 4.1666666666666667e-02f);       // 1/4!
    p = jx_fma(p, r, 1.6666666666666667e-01f);       // 1/3!
    p = jx_fma(p, r, 0.5f);
    p = jx_fma(p, r, 1.0f);
    p = jx_fma(p, r, 1.0f);
    const int ni{static_cast<int>(n)};
    return p * u2f(static_cast<std::uint32_t>(ni + 127) << 23);
}

// Cube root of a positive normal x: Newton iterations for x^(-1/3) from a
// bit-pattern seed within a few percent (quadratic convergence: three reach
// float precision), then one Newton correction of x^(1/3) itself. At most
// 0.72 ulp on the XYB domain.
JX_HD float jx_cbrt(float x) {
    const std::uint32_t u{f2u(x)};
    float r{u2f(0x54a2fa8cu - u / 3u)};  // seed for x^(-1/3), within a few percent
    for (int it{0}; it < 3; ++it) {
        const float t{(r * r) * r};
        const float e{jx_fma(-x, t, 1.0f)};
        r = jx_fma(r * 0.333333343f, e, r);
    }
    float y{(x * r) * r};
    const float y2{y * y};
    const float res{jx_fma(y2, y, -x)};
    y = jx_fma(-res, (r * r) * 0.333333343f, y);
    return y;
}

// x^2.4 for positive normal x, as x^2 * x^0.4 with x = 2^k m, m in [1, 2)
// and k = 5q + r (r in 0..4): x^0.4 = 2^(2q) * 2^(0.4 r) * m^0.4. m^0.4 is a
// degree-8 polynomial in m - 1.5 (Chebyshev interpolation of m^0.4 at 200
// nodes on [1, 2], converted to powers and rounded to float; relative error
// 8e-8 in float evaluation). At most 2.6 ulp on (0.09, 1], and 1 maps to 1.
JX_HD float jx_pow24(float x) {
    const std::uint32_t u{f2u(x)};
    const int k{static_cast<int>((u >> 23) & 0xffu) - 127};
    const float m{u2f((u & 0x7fffffu) | 0x3f800000u)};
    const int q{(k >= 0 ? k : k - 4) / 5};  // floor(k / 5)
    const int r{k - 5 * q};
    const float c{r == 0 ? 1.0f
                         : (r == 1 ? 1.31950791077289425f
                                   : (r == 2 ? 1.74110112659224828f
                                             : (r == 3 ? 2.29739670999407037f : 3.03143313302079624f)))};
    const float v{m - 1.5f};  // exact
    float p{-8.58357804e-04f};
    p = jx_fma(p, v, 1.51637842e-03f);
    p = jx_fma(p, v, -2.33355959e-03f);
    p = jx_fma(p, v, 4.58948039e-03f);
    p = jx_fma(p, v, -9.66759456e-03f);
    p = jx_fma(p, v, 2.23054436e-02f);
    p = jx_fma(p, v, -6.27241061e-02f);
    p = jx_fma(p, v, 3.13621006e-01f);
    p = jx_fma(p, v, 1.17607902e+00f);
    return ((x * x) * (p * c)) * u2f(static_cast<std::uint32_t>(2 * q + 127) << 23);
}

}  // namespace jxb
