/* CPU restatement of the encoder frontend (test infrastructure: the checker
 * for the CUDA frontend and the CPU baseline; never part of the product).
 *
 * Restates, per 64x64 colour tile, the device-only stages of the reference
 * encoder m-pilia/cujpegxl:
 *   NV12 -> XYB ............ src/xyb_impl.cuh:37-70, src/frontend_fused.cu:214-230
 *   adaptive quant field ... src/frontend_fused.cu:54-204, src/adaptive_quant_impl.cuh:30-116,
 *                            constants src/frontend_fused.cu:349-380
 *   inverse gaborish ....... src/frontend_transform.cu:19-49, src/gaborish.h
 *   transform selection .... src/transform_select_impl.cuh:49-201 (host twin arithmetic)
 *   variable DCT ........... src/frontend_transform.cu:66-159
 *   chroma from luma ....... src/frontend_quantize.cu:49-118, src/cfl.h:36-80
 *   quantisation ........... src/frontend_quantize.cu:125-201, src/vardct_layout.h:88-111
 *   calibration ............ src/quant_calibration.h:49-88
 * with the float-operation contract of the product (explicit fmaf where the
 * product fuses, plain rounded operations elsewhere, deterministic
 * transcendentals, the partial-sum and reduction orders of the reference), so
 * results are bit-identical to the GPU path. Compile with -ffp-contract=off.
 *
 * Chroma is upsampled with the exact bilinear weights of the reference's CUDA
 * texture fetch at ((x+0.5)/2, (y+0.5)/2); the reference's tests accept the
 * texture unit's 1/256 weight quantisation as a tolerance (its
 * tests/xyb_conformance_test.py:6-9), with the weights here exactly 1/4, 3/4.
 */

#include <math.h>
#include <pthread.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

/* ---- deterministic math (same methods as the product's jxl_math.cuh) ---- */

static uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

float oracle_log2(float x) {
    uint32_t u = f2u(x);
    int e = (int)((u >> 23) & 0xffu) - 127;
    float m = u2f((u & 0x7fffffu) | 0x3f800000u);
    if (m > 1.41421356f) { m = m * 0.5f; e += 1; }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float s2 = s * s;
    float p = 0.32059889797532520f;
    p = fmaf(p, s2, 0.41219858311113244f);
    p = fmaf(p, s2, 0.57707801635558536f);
    p = fmaf(p, s2, 0.96179669392597560f);
    p = fmaf(p, s2, 2.88539008177792681f);
    return (float)e + s * p;
}

float oracle_exp2(float y) {
    const float n = rintf(y);
    const float f = y - n;
    float p = 1.3215486790144307e-06f;
    p = fmaf(p, f, 1.5252733804059840e-05f);
    p = fmaf(p, f, 1.5403530393381609e-04f);
    p = fmaf(p, f, 1.3333558146428443e-03f);
    p = fmaf(p, f, 9.6181291076284772e-03f);
    p = fmaf(p, f, 5.5504108664821580e-02f);
    p = fmaf(p, f, 2.4022650695910071e-01f);
    p = fmaf(p, f, 6.9314718055994531e-01f);
    p = fmaf(p, f, 1.0f);
    return p * u2f((uint32_t)((int)n + 127) << 23);
}

float oracle_exp(float x) {
    const float n = rintf(x * 1.44269504088896341f);
    float r = fmaf(-n, 0.693145751953125f, x);
    r = fmaf(-n, 1.42860682030941723e-06f, r);
    float p = 2.4801587301587302e-05f;
    p = fmaf(p, r, 1.9841269841269841e-04f);
    p = fmaf(p, r, 1.3888888888888889e-03f);
    p = fmaf(p, r, 8.3333333333333333e-03f);
    p = fmaf(p, r, 4.1666666666666667e-02f);
    p = fmaf(p, r, 1.6666666666666667e-01f);
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    return p * u2f((uint32_t)((int)n + 127) << 23);
}

float oracle_cbrt(float x) {
    const uint32_t u = f2u(x);
    float r = u2f(0x54a2fa8cu - u / 3u);
    for (int it = 0; it < 3; ++it) {
        const float t = (r * r) * r;
        const float e = fmaf(-x, t, 1.0f);
        r = fmaf(r * 0.333333343f, e, r);
    }
    float y = (x * r) * r;
    const float y2 = y * y;
    const float res = fmaf(y2, y, -x);
    y = fmaf(-res, (r * r) * 0.333333343f, y);
    return y;
}

float oracle_pow24(float x) {
    const uint32_t u = f2u(x);
    const int k = (int)((u >> 23) & 0xffu) - 127;
    const float m = u2f((u & 0x7fffffu) | 0x3f800000u);
    const int q = (k >= 0 ? k : k - 4) / 5;
    const int r = k - 5 * q;
    const float c = r == 0 ? 1.0f
                           : (r == 1 ? 1.31950791077289425f
                                     : (r == 2 ? 1.74110112659224828f
                                               : (r == 3 ? 2.29739670999407037f : 3.03143313302079624f)));
    const float v = m - 1.5f;
    float p = -8.58357804e-04f;
    p = fmaf(p, v, 1.51637842e-03f);
    p = fmaf(p, v, -2.33355959e-03f);
    p = fmaf(p, v, 4.58948039e-03f);
    p = fmaf(p, v, -9.66759456e-03f);
    p = fmaf(p, v, 2.23054436e-02f);
    p = fmaf(p, v, -6.27241061e-02f);
    p = fmaf(p, v, 3.13621006e-01f);
    p = fmaf(p, v, 1.17607902e+00f);
    return ((x * x) * (p * c)) * u2f((uint32_t)(2 * q + 127) << 23);
}

/* IEEE binary16 conversions (round to nearest even). */
uint16_t oracle_f2h(float f) {
    const uint32_t u = f2u(f);
    const uint32_t sign = (u >> 16) & 0x8000u;
    const uint32_t a = u & 0x7fffffffu;
    if (a >= 0x7f800000u) return (uint16_t)(sign | (a > 0x7f800000u ? 0x7e00u : 0x7c00u));
    if (a >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);
    if (a >= 0x38800000u) {
        const uint32_t mant = a & 0x7fffffu;
        uint32_t h = ((((a >> 23) - 127u + 15u)) << 10) | (mant >> 13);
        const uint32_t rem = mant & 0x1fffu;
        if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h++;
        return (uint16_t)(sign | h);
    }
    if (a < 0x33000000u) return (uint16_t)sign;
    const uint32_t exp = a >> 23;
    const uint32_t mant = (a & 0x7fffffu) | 0x800000u;
    const uint32_t shift = 126u - exp;
    uint32_t h = mant >> shift;
    const uint32_t rem = mant & ((1u << shift) - 1u);
    const uint32_t halfway = 1u << (shift - 1u);
    if (rem > halfway || (rem == halfway && (h & 1u))) h++;
    return (uint16_t)(sign | h);
}

float oracle_h2f(uint16_t h) {
    const uint32_t sign = ((uint32_t)h & 0x8000u) << 16;
    const uint32_t e = ((uint32_t)h >> 10) & 0x1fu;
    const uint32_t m = (uint32_t)h & 0x3ffu;
    if (e == 0) {
        const float v = (float)m * 5.9604644775390625e-8f;
        return sign ? -v : v;
    }
    if (e == 31) return u2f(sign | 0x7f800000u | (m << 13));
    return u2f(sign | ((e - 15u + 127u) << 23) | (m << 13));
}

/* ---- constants (values of the reference encoder) ---- */

#define M00 0.30f
#define M02 0.078f
#define M01 (1.0f - M02 - M00)
#define M10 0.23f
#define M12 0.078f
#define M11 (1.0f - M12 - M10)
#define M20 0.24342268924547819f
#define M21 0.20476744424496821f
#define M22 (1.0f - M20 - M21)
#define OPSIN_BIAS 0.0037930732552754493f
#define NEG_CBRT_BIAS (-0.15595419704914093f)
#define CR_TO_R 1.5748f
#define CB_TO_G 0.1873242729f
#define CR_TO_G 0.4681242729f
#define CB_TO_B 1.8556f

static const float kChromaCenter = 128.0f / 255.0f;
static const float kInv255 = 1.0f / 255.0f;

static const float GK0 = -0.09495815671340026f;
static const float GK1 = -0.041031725066768575f;
static const float GK2 = 0.013710004822696948f;
static const float GK3 = 0.006510206083837737f;
static const float GK4 = -0.0014789063378272242f;

#define SG_MUL 226.77216153508914f
#define SG_MUL2 (1.0f / 73.377132366608819f)
#define SG_LOG2 0.693147181f
#define SG_RET_MUL (SG_MUL2 * 18.6580932135f * SG_LOG2)
#define SG_VOFF 7.7825991679894591f

static float g_gab[6];          /* centre, edge, edge2, diag, knight, diag2 */
static float g_ratio_num, g_ratio_voff, g_ratio_den;
static float g_mask_sqrt;
static float g_sel_basis[3][1024];
static float g_dct_basis[3][1024];
static float g_sel_w[3][1024];
static float g_deq[3][3][1024];
static float* g_l2;             /* log2f(1 + i) */
static double g_ob[2][16];
static int g_ready;
static pthread_once_t g_once = PTHREAD_ONCE_INIT;

#define LOG2_TABLE (1 << 19)

#include "../cujpegxl_b200/csrc/jxl_dequant_tables.inc"

static void init_tables(void) {
    /* Gaborish weights as the float constant expressions of src/gaborish.h:21-28. */
    const float nm = 1.0f / (1.0f + 4.0f * (GK0 + GK1 + GK2 + GK4 + 2.0f * GK3));
    g_gab[0] = nm; g_gab[1] = nm * GK0; g_gab[2] = nm * GK2;
    g_gab[3] = nm * GK1; g_gab[4] = nm * GK3; g_gab[5] = nm * GK4;
    g_ratio_num = SG_RET_MUL * 3.0f * SG_MUL;
    g_ratio_voff = SG_VOFF * SG_LOG2 + 1e-2f;
    g_ratio_den = SG_LOG2 * SG_MUL;
    g_mask_sqrt = sqrtf(211.66567973503678f * 1e8f);
    for (int si = 0; si < 3; ++si) {
        const int n = 8 << si;
        for (int k = 0; k < n; ++k) {
            const double g = k == 0 ? 1.0 / n : 1.4142135623730950488 / n;
            const float gf = k == 0 ? 1.0f / n : 1.4142135623730951f / n;
            for (int t = 0; t < n; ++t) {
                g_sel_basis[si][k * n + t] = (float)(g * cos(3.14159265358979323846 * (t + 0.5) * k / n));
                const float arg = 3.14159265358979323846f * (t + 0.5f) * k / n;
                g_dct_basis[si][k * n + t] = gf * cosf(arg);
            }
        }
    }
    for (int c = 0; c < 3; ++c) {
        memcpy(g_deq[0][c], kDequantBits8[c], 64 * 4);
        memcpy(g_deq[1][c], kDequantBits16[c], 256 * 4);
        memcpy(g_deq[2][c], kDequantBits32[c], 1024 * 4);
    }
    for (int si = 0; si < 3; ++si) {
        const int n = 8 << si;
        for (int fx = 0; fx < n; ++fx) {
            for (int fy = 0; fy < n; ++fy) {
                int sx = (int)lround(fx * 8.0 / n);
                int sy = (int)lround(fy * 8.0 / n);
                sx = sx > 7 ? 7 : sx;
                sy = sy > 7 ? 7 : sy;
                g_sel_w[si][fx * n + fy] = g_deq[0][1][sx * 8 + sy];
            }
        }
    }
    g_l2 = (float*)malloc(sizeof(float) * LOG2_TABLE);
    for (int i = 0; i < LOG2_TABLE; ++i) g_l2[i] = log2f(1.0f + (float)i);
    for (int mi = 0; mi < 2; ++mi) {
        const int m = mi == 0 ? 2 : 4;
        const double md = (double)m;
        for (int k = 0; k < m; ++k) {
            for (int nn = 0; nn < m; ++nn) {
                const double nv = k == 0 ? sqrt(1.0 / md) : sqrt(2.0 / md);
                g_ob[mi][k * 4 + nn] = nv * cos(3.14159265358979323846 * ((double)nn + 0.5) * (double)k / md);
            }
        }
    }
    g_ready = 1;
}

static void ensure_tables(void) { pthread_once(&g_once, init_tables); }

/* ---- calibration (src/quant_calibration.h:49-88) and AQ scalars ---- */

void oracle_scalars(float distance, OracleScalars* s) {
    const float quant_ac = 0.725f / distance;
    float pw = 0.3f * powf((1.0f / 0.3f) * distance, 0.83f);
    float mn = distance < pw ? distance : pw;
    const float bt_dc = 0.5f * distance > mn ? 0.5f * distance : mn;
    float qdcf = 1.095924047623553f / bt_dc;
    qdcf = qdcf < 50.0f ? qdcf : 50.0f;
    float scale = 65536.0f * quant_ac / 5.0f;
    if (scale < 1.0f) scale = 1.0f;
    if (scale > 32768.0f) scale = 32768.0f;
    int gs = (int)scale;
    const int sqdc = (int)(qdcf * 4096 * 1.6f);
    if (gs > sqdc) gs = sqdc <= 0 ? 1 : sqdc;
    const float inv_gs = 1.0f * 65536.0f / (float)gs;
    float fval = qdcf * inv_gs + 0.5f;
    fval = fval < 65536.0f ? fval : 65536.0f;
    const int qdc = (int)fval;
    int q = (int)lroundf(quant_ac * inv_gs);
    q = q < 1 ? 1 : (q > 256 ? 256 : q);
    const float gsf = (float)gs * (1.0f / 65536);
    s->global_scale = (uint32_t)gs;
    s->quant_dc = (uint32_t)qdc;
    s->raw_quant_field = (uint32_t)q;
    s->gsf = gsf;
    s->inv_global_scale = inv_gs;
    s->qgsf_select = (float)q * gsf;
    s->dc_scale = gsf * (float)qdc;

    const float ascale = 0.725f / distance;
    const float base_level = 0.48f * ascale;
    float dampen = 1.0f;
    if (distance >= 2.0f) {
        dampen = 1.0f - (distance - 2.0f) / (14.0f - 2.0f);
        if (dampen < 0.0f) dampen = 0.0f;
    }
    s->mul_pb = ascale * dampen;
    s->add_pb = (1.0f - dampen) * base_level;
    const float efm = distance < 2.0f ? (2.0f - distance) * 0.5f : 0.0f;
    const float km0 = 0.125f;
    const float km1 = 0.10f - efm * 0.10f;
    const float km2 = 0.09f - efm * 0.09f;
    const float km3 = 0.06f - efm * 0.06f;
    const float norm = 0.29959705784054957f / (km0 + km1 + km2 + km3);
    s->km[0] = km0 * norm;
    s->km[1] = km1 * norm;
    s->km[2] = km2 * norm;
    s->km[3] = km3 * norm;
}

/* ---- per-pixel stages ---- */

static float clamp01(float v) { return fminf(fmaxf(v, 0.0f), 1.0f); }

static float srgb_to_linear(float e) {
    return e <= 0.04045f ? e * (1.0f / 12.92f) : oracle_pow24((e + 0.055f) * (1.0f / 1.055f));
}

static void xyb_pixel(const OracleFrame* in, int gx, int gy, float* ox, float* oy, float* ob) {
    const float yv = (float)in->luma[(size_t)gy * in->luma_pitch + gx] * kInv255;
    const int cw = in->width >> 1, ch = in->height >> 1;
    const int jx = gx >> 1, jy = gy >> 1;
    int xa, xb, wxa, wxb, ya, yb, wya, wyb;
    if (gx & 1) { xa = jx; xb = jx + 1 < cw ? jx + 1 : cw - 1; wxa = 3; wxb = 1; }
    else { xa = jx - 1 > 0 ? jx - 1 : 0; xb = jx; wxa = 1; wxb = 3; }
    if (gy & 1) { ya = jy; yb = jy + 1 < ch ? jy + 1 : ch - 1; wya = 3; wyb = 1; }
    else { ya = jy - 1 > 0 ? jy - 1 : 0; yb = jy; wya = 1; wyb = 3; }
    const uint8_t* ra = in->chroma + (size_t)ya * in->chroma_pitch;
    const uint8_t* rb = in->chroma + (size_t)yb * in->chroma_pitch;
    const int scb = wya * (wxa * ra[2 * xa] + wxb * ra[2 * xb]) + wyb * (wxa * rb[2 * xa] + wxb * rb[2 * xb]);
    const int scr = wya * (wxa * ra[2 * xa + 1] + wxb * ra[2 * xb + 1]) +
                    wyb * (wxa * rb[2 * xa + 1] + wxb * rb[2 * xb + 1]);
    const float cb = (float)scb / 4080.0f - kChromaCenter;
    const float cr = (float)scr / 4080.0f - kChromaCenter;
    const float r = clamp01(srgb_to_linear(clamp01(fmaf(CR_TO_R, cr, yv))));
    const float g = clamp01(srgb_to_linear(clamp01(fmaf(-CR_TO_G, cr, fmaf(-CB_TO_G, cb, yv)))));
    const float b = clamp01(srgb_to_linear(clamp01(fmaf(CB_TO_B, cb, yv))));
    float m0 = fmaf(M02, b, fmaf(M01, g, M00 * r)) + OPSIN_BIAS;
    float m1 = fmaf(M12, b, fmaf(M11, g, M10 * r)) + OPSIN_BIAS;
    float m2 = fmaf(M22, b, fmaf(M21, g, M20 * r)) + OPSIN_BIAS;
    m0 = oracle_cbrt(fmaxf(m0, 0.0f)) + NEG_CBRT_BIAS;
    m1 = oracle_cbrt(fmaxf(m1, 0.0f)) + NEG_CBRT_BIAS;
    m2 = oracle_cbrt(fmaxf(m2, 0.0f)) + NEG_CBRT_BIAS;
    *ox = 0.5f * (m0 - m1);
    *oy = 0.5f * (m0 + m1);
    *ob = m2;
}

void oracle_xyb_pixel(const OracleFrame* in, int gx, int gy, float* out3) {
    ensure_tables();
    xyb_pixel(in, gx, gy, &out3[0], &out3[1], &out3[2]);
}

static float ratio_gamma(float v, int invert) {
    v = v < 0.0f ? 0.0f : v;
    const float v2 = v * v;
    const float num = fmaf(g_ratio_num, v2, 1e-2f);
    const float den = fmaf(g_ratio_den * v, v2, g_ratio_voff);
    return invert ? num / den : den / num;
}

static float masking_sqrt(float v) { return 0.25f * sqrtf(fmaf(v, g_mask_sqrt, 27.505837037000106f)); }

static float compute_mask(float out_val) {
    const float v1 = fmaxf(out_val * 0.80061762862741759f, 1e-3f);
    const float v2 = 1.0f / (v1 + 302.59587815579727f);
    const float v3 = 1.0f / fmaf(v1, v1, 3.7179635626140772f);
    const float v4 = 1.0f / fmaf(v1, v1, 0.25f * 3.7179635626140772f);
    float r = fmaf(9.4708735624378946f, v4, -0.7647f);
    r = fmaf(17.35036561631863f, v2, r);
    r = fmaf(6.7943250517376494f, v3, r);
    return r;
}

static void swap_if(float* a, float* b) { if (*a > *b) { const float t = *a; *a = *b; *b = t; } }

static void keep_min4(float v, float* m) {
    if (v < m[3]) {
        if (v < m[0]) { m[3] = m[2]; m[2] = m[1]; m[1] = m[0]; m[0] = v; }
        else if (v < m[1]) { m[3] = m[2]; m[2] = m[1]; m[1] = v; }
        else if (v < m[2]) { m[3] = m[2]; m[2] = v; }
        else { m[3] = v; }
    }
}

static float erosion_cell(const float* pre, int sx0, int sy0, int cx, int cy, const float* km) {
    const int xm = cx > 0 ? cx - 1 : cx, xp = cx + 1 < 8 ? cx + 1 : cx;
    const int ym = cy > 0 ? cy - 1 : cy, yp = cy + 1 < 8 ? cy + 1 : cy;
#define AT(x, y) pre[(sy0 + (y)) * 16 + sx0 + (x)]
    float m[4] = {AT(cx, cy), AT(xm, cy), AT(xp, cy), AT(xm, ym)};
    swap_if(&m[0], &m[1]); swap_if(&m[0], &m[2]); swap_if(&m[0], &m[3]);
    swap_if(&m[1], &m[2]); swap_if(&m[1], &m[3]); swap_if(&m[2], &m[3]);
    keep_min4(AT(cx, ym), m); keep_min4(AT(xp, ym), m); keep_min4(AT(xm, yp), m);
    keep_min4(AT(cx, yp), m); keep_min4(AT(xp, yp), m);
#undef AT
    float r = km[0] * m[0];
    r = fmaf(km[1], m[1], r);
    r = fmaf(km[2], m[2], r);
    r = fmaf(km[3], m[3], r);
    return r;
}

/* Sum of 32 values with the pairing of a shfl_down reduction (16, 8, 4, 2, 1). */
static float tree32(float* v) {
    for (int off = 16; off > 0; off >>= 1)
        for (int i = 0; i < off; ++i) v[i] = v[i] + v[i + off];
    return v[0];
}

/* ---- tile processing ---- */

void oracle_dc_from_llf(int m, const float* llf, float* dc);
void oracle_cfl_maps(float sxy, float syy, float sby, int* mx, int* mb);

#define XS 68
#define XP (XS * XS)
#define SS 65
#define SP (64 * SS)

typedef struct {
    float xyb[3 * XP];
    float shp[3 * SP];
    float pre[256];
    float cost8[64], cost16[16], cost32[4];
    int qf[64];
    signed char acs[64];
    unsigned char owner[64];
    int nz[3][64];
    uint16_t coef[3][64 * 64];
} Tile;

/* Separable selection cost of one NxN block at tile-local pixel (x0, y0) with
 * the host twin's arithmetic: per-coefficient contributions, partials over
 * e = t, t+256, ... and a power-of-two tree (src/transform_select_impl.cuh:49-115). */
static float sel_cost(const float* SY, int x0, int y0, int n, float qgsf) {
    const int si = n == 8 ? 0 : (n == 16 ? 1 : 2);
    const float* B = g_sel_basis[si];
    float rows[1024], cd[1024], cr[1024];
    for (int fx = 0; fx < n; ++fx)
        for (int r = 0; r < n; ++r) {
            float s = 0.0f;
            for (int c = 0; c < n; ++c) s = s + B[fx * n + c] * SY[(y0 + r) * SS + x0 + c];
            rows[fx * n + r] = s;
        }
    const int m = n / 8;
    for (int fx = 0; fx < n; ++fx)
        for (int fy = 0; fy < n; ++fy) {
            const int e = fx * n + fy;
            float coeff = 0.0f;
            for (int r = 0; r < n; ++r) coeff = coeff + B[fy * n + r] * rows[fx * n + r];
            float d = 0.0f, rt = 0.0f;
            if (!(fx < m && fy < m)) {
                const float w = g_sel_w[si][e];
                const float q = rintf((coeff * qgsf) / w);
                const float err = (q * w) / qgsf - coeff;
                d = err * err;
                if (q != 0.0f) {
                    int a = (int)fabsf(q);
                    a = a < LOG2_TABLE ? a : LOG2_TABLE - 1;
                    rt = 1.0f + g_l2[a];
                }
            }
            cd[e] = d;
            cr[e] = rt;
        }
    float pd[256], pr[256];
    for (int t = 0; t < 256; ++t) {
        float d = 0.0f, r = 0.0f;
        for (int e = t; e < n * n; e += 256) { d = d + cd[e]; r = r + cr[e]; }
        pd[t] = d;
        pr[t] = r;
    }
    for (int s = 128; s > 0; s >>= 1)
        for (int t = 0; t < s; ++t) { pd[t] = pd[t] + pd[t + s]; pr[t] = pr[t] + pr[t + s]; }
    return (float)(n * n) * pd[0] + 6.0e-4f * pr[0];
}

static void process_tile(const OracleFrame* in, const OracleScalars* sc, const OracleOutputs* out,
                         int tx, int ty, Tile* T) {
    const int W = in->width, H = in->height;
    const int bw = W >> 3, bh = H >> 3;
    const size_t nblocks = (size_t)bw * bh;
    const int px0 = tx * 64, py0 = ty * 64, bx0 = tx * 8, by0 = ty * 8;
    const int cmw = (bw + 7) / 8;

    /* 1. XYB with a 2-pixel halo at clamped coordinates. */
    for (int ly = 0; ly < XS; ++ly)
        for (int lx = 0; lx < XS; ++lx) {
            int gx = px0 - 2 + lx, gy = py0 - 2 + ly;
            gx = gx < 0 ? 0 : (gx > W - 1 ? W - 1 : gx);
            gy = gy < 0 ? 0 : (gy > H - 1 ? H - 1 : gy);
            xyb_pixel(in, gx, gy, &T->xyb[ly * XS + lx], &T->xyb[XP + ly * XS + lx],
                      &T->xyb[2 * XP + ly * XS + lx]);
        }
    if (out->dbg_xyb)
        for (int c = 0; c < 3; ++c)
            for (int y = 0; y < 64 && py0 + y < H; ++y)
                for (int x = 0; x < 64 && px0 + x < W; ++x)
                    out->dbg_xyb[((size_t)c * H + py0 + y) * W + px0 + x] = T->xyb[c * XP + (y + 2) * XS + x + 2];

    /* 2. adaptive quantisation. */
    const float* Y = T->xyb + XP;
    for (int ci = 0; ci < 256; ++ci) {
        const int ccx = ci & 15, ccy = ci >> 4;
        float sum = 0.0f;
        for (int dy = 0; dy < 4; ++dy)
            for (int dx = 0; dx < 4; ++dx) {
                const int ix = ccx * 4 + dx + 2, iy = ccy * 4 + dy + 2;
                const float yv = Y[iy * XS + ix];
                const float base = 0.25f * (((Y[(iy + 1) * XS + ix] + Y[(iy - 1) * XS + ix]) + Y[iy * XS + ix - 1]) +
                                            Y[iy * XS + ix + 1]);
                float d = ratio_gamma(yv + 0.019f, 0) * (yv - base);
                d = d * d;
                d = fminf(d, 0.2f);
                sum = sum + masking_sqrt(d);
            }
        T->pre[ci] = 0.25f * sum;
    }
    const float kLimit = 0.027121074570634722f;
    for (int lb = 0; lb < 64; ++lb) {
        const int lbx = lb & 7, lby = lb >> 3;
        if (bx0 + lbx >= bw || by0 + lby >= bh) continue;
        float red[2][4];
        for (int half = 0; half < 2; ++half) {
            float hv[32], gv[32], bvv[32], ev[32];
            for (int lane = 0; lane < 32; ++lane) {
                const int fx = lane & 7, fy = (lane >> 3) + 4 * half;
                const int ix = lbx * 8 + fx + 2, iy = lby * 8 + fy + 2;
                const float yv = Y[iy * XS + ix];
                const float xv = T->xyb[iy * XS + ix];
                const float bv = T->xyb[2 * XP + iy * XS + ix];
                float hf = 0.0f;
                if (fx < 7) hf = hf + fminf(0.0206f, fabsf(yv - Y[iy * XS + ix + 1]));
                if (fy < 7) hf = hf + fminf(0.0206f, fabsf(yv - Y[(iy + 1) * XS + ix]));
                const float iny = yv + 0.16f;
                const float gp = ratio_gamma(iny - xv, 1) + ratio_gamma(iny + xv, 1);
                const float pye = (yv + 0.084381641171960495f) + fabsf(xv);
                const float bp = bv > pye ? fminf(bv - pye, kLimit) : 0.0f;
                float er = 0.0f;
                if (half == 0 && lane < 4)
                    er = erosion_cell(T->pre, (lbx >> 2) * 8, (lby >> 2) * 8, 2 * (lbx & 3) + (lane & 1),
                                      2 * (lby & 3) + (lane >> 1), sc->km);
                hv[lane] = hf; gv[lane] = gp; bvv[lane] = bp; ev[lane] = er;
            }
            red[half][0] = tree32(hv);
            red[half][1] = tree32(gv);
            red[half][2] = tree32(bvv);
            red[half][3] = tree32(ev);
        }
        const float hf_sum = red[0][0] + red[1][0];
        const float gamma_overall = (red[0][1] + red[1][1]) * (0.5f / 64.0f);
        float blue_sum = red[0][2] + red[1][2];
        const float aq = red[0][3] + red[1][3];
        if (blue_sum >= 32.0f * kLimit) blue_sum = 64.0f * kLimit - blue_sum;
        const float maxl = 15.398788439047934f * kLimit;
        if (blue_sum >= maxl) blue_sum = maxl;
        float ov = compute_mask(aq);
        ov = ov + fmaf(hf_sum, -0.38f, 0.42f);
        ov = fmaf(0.1005613337192697f, oracle_log2(gamma_overall), ov);
        ov = fmaf(blue_sum, 0.14207000358439159f, ov);
        const float qval = fmaf(oracle_exp(ov), sc->mul_pb, sc->add_pb);
        int qi = (int)fmaf(qval, sc->inv_global_scale, 0.5f);
        qi = qi < 1 ? 1 : (qi > 256 ? 256 : qi);
        T->qf[lb] = qi;
    }

    /* 3. inverse gaborish. */
    for (int c = 0; c < 3; ++c)
        for (int y = 0; y < 64; ++y)
            for (int x = 0; x < 64; ++x) {
                const float* P = T->xyb + c * XP + (y + 2) * XS + x + 2;
#define A(dx, dy) P[(dy) * XS + (dx)]
                const float e = ((A(-1, 0) + A(1, 0)) + A(0, -1)) + A(0, 1);
                const float r2 = ((A(-2, 0) + A(2, 0)) + A(0, -2)) + A(0, 2);
                const float dg = ((A(-1, -1) + A(1, -1)) + A(-1, 1)) + A(1, 1);
                const float l8 = ((((((A(-2, -1) + A(2, -1)) + A(-2, 1)) + A(2, 1)) + A(-1, -2)) + A(1, -2)) +
                                  A(-1, 2)) + A(1, 2);
                const float d4 = ((A(-2, -2) + A(2, -2)) + A(-2, 2)) + A(2, 2);
                float s = g_gab[0] * A(0, 0);
#undef A
                s = fmaf(g_gab[1], e, s);
                s = fmaf(g_gab[2], r2, s);
                s = fmaf(g_gab[3], dg, s);
                s = fmaf(g_gab[4], l8, s);
                s = fmaf(g_gab[5], d4, s);
                T->shp[c * SP + y * SS + x] = s;
            }
    if (out->dbg_sharp)
        for (int c = 0; c < 3; ++c)
            for (int y = 0; y < 64 && py0 + y < H; ++y)
                for (int x = 0; x < 64 && px0 + x < W; ++x)
                    out->dbg_sharp[((size_t)c * H + py0 + y) * W + px0 + x] = T->shp[c * SP + y * SS + x];

    /* 4. transform selection. */
    const float* SY = T->shp + SP;
    for (int lb = 0; lb < 64; ++lb)
        if (bx0 + (lb & 7) < bw && by0 + (lb >> 3) < bh)
            T->cost8[lb] = sel_cost(SY, (lb & 7) * 8, (lb >> 3) * 8, 8, sc->qgsf_select);
    for (int qd = 0; qd < 16; ++qd)
        if (bx0 + 2 * (qd & 3) + 2 <= bw && by0 + 2 * (qd >> 2) + 2 <= bh)
            T->cost16[qd] = sel_cost(SY, (qd & 3) * 16, (qd >> 2) * 16, 16, sc->qgsf_select);
    for (int ri = 0; ri < 4; ++ri)
        if (bx0 + 4 * (ri & 1) + 4 <= bw && by0 + 4 * (ri >> 1) + 4 <= bh)
            T->cost32[ri] = sel_cost(SY, (ri & 1) * 32, (ri >> 1) * 32, 32, sc->qgsf_select);
    for (int ri = 0; ri < 4; ++ri) {
        const int rlx = (ri & 1) * 4, rly = (ri >> 1) * 4;
        const int rbx = bx0 + rlx, rby = by0 + rly;
        if (rbx >= bw || rby >= bh) continue;
        const float INF = 1.0e30f;
        const int fit32 = rbx + 4 <= bw && rby + 4 <= bh;
        const float c32 = fit32 ? T->cost32[ri] : INF;
        float split = 0.0f;
        int choice[2][2];
        for (int qy = 0; qy < 2; ++qy)
            for (int qx = 0; qx < 2; ++qx) {
                const int bx = rbx + 2 * qx, by = rby + 2 * qy;
                float sum8 = 0.0f;
                int any = 0;
                for (int dy = 0; dy < 2; ++dy)
                    for (int dx = 0; dx < 2; ++dx)
                        if (bx + dx < bw && by + dy < bh) {
                            sum8 = sum8 + T->cost8[(rly + 2 * qy + dy) * 8 + rlx + 2 * qx + dx];
                            any = 1;
                        }
                if (!any) { choice[qy][qx] = -1; continue; }
                const int fit16 = bx + 2 <= bw && by + 2 <= bh;
                const float c16 = fit16 ? T->cost16[((rly >> 1) + qy) * 4 + (rlx >> 1) + qx] : INF;
                if (fit16 && c16 <= sum8 + 1.0e-6f) { choice[qy][qx] = 16; split = split + c16; }
                else { choice[qy][qx] = 8; split = split + sum8; }
            }
        if (fit32 && c32 <= split + 1.0e-6f) {
            for (int dy = 0; dy < 4; ++dy)
                for (int dx = 0; dx < 4; ++dx) T->acs[(rly + dy) * 8 + rlx + dx] = (dx == 0 && dy == 0) ? 32 : 0;
        } else {
            for (int qy = 0; qy < 2; ++qy)
                for (int qx = 0; qx < 2; ++qx) {
                    const int chs = choice[qy][qx];
                    if (chs < 0) continue;
                    for (int dy = 0; dy < 2; ++dy)
                        for (int dx = 0; dx < 2; ++dx) {
                            const int l = (rly + 2 * qy + dy) * 8 + rlx + 2 * qx + dx;
                            if (chs == 16) T->acs[l] = (dx == 0 && dy == 0) ? 16 : 0;
                            else if (rbx + 2 * qx + dx < bw && rby + 2 * qy + dy < bh) T->acs[l] = 8;
                        }
                }
        }
    }
    memset(T->owner, 255, sizeof(T->owner));
    for (int lb = 0; lb < 64; ++lb) {
        if (bx0 + (lb & 7) >= bw || by0 + (lb >> 3) >= bh || T->acs[lb] == 0) continue;
        const int s = T->acs[lb] >> 3;
        for (int dy = 0; dy < s; ++dy)
            for (int dx = 0; dx < s; ++dx) T->owner[lb + dy * 8 + dx] = (unsigned char)lb;
    }

    /* 5. variable DCT -> FP16 in the tile's covered-block layout. */
    for (int lb = 0; lb < 64; ++lb) {
        if (bx0 + (lb & 7) >= bw || by0 + (lb >> 3) >= bh || T->acs[lb] == 0) continue;
        const int n = T->acs[lb];
        const int si = n == 8 ? 0 : (n == 16 ? 1 : 2);
        const float* B = g_dct_basis[si];
        const int side = n >> 3;
        for (int c = 0; c < 3; ++c) {
            const float* P = T->shp + c * SP;
            float rows[1024];
            for (int fx = 0; fx < n; ++fx)
                for (int r = 0; r < n; ++r) {
                    float s = 0.0f;
                    for (int col = 0; col < n; ++col)
                        s = fmaf(B[fx * n + col], P[((lb >> 3) * 8 + r) * SS + (lb & 7) * 8 + col], s);
                    rows[fx * n + r] = s;
                }
            for (int fx = 0; fx < n; ++fx)
                for (int fy = 0; fy < n; ++fy) {
                    float coeff = 0.0f;
                    for (int r = 0; r < n; ++r) coeff = fmaf(B[fy * n + r], rows[fx * n + r], coeff);
                    const int raw = fx * n + fy, q = raw >> 6;
                    const int l = lb + (q / side) * 8 + q % side;
                    T->coef[c][l * 64 + (raw & 63)] = oracle_f2h(coeff);
                }
        }
    }
    if (out->dbg_coeff)
        for (int c = 0; c < 3; ++c)
            for (int lb = 0; lb < 64; ++lb) {
                const int gbx = bx0 + (lb & 7), gby = by0 + (lb >> 3);
                if (gbx >= bw || gby >= bh) continue;
                memcpy(out->dbg_coeff + (size_t)c * nblocks * 64 + ((size_t)gby * bw + gbx) * 64,
                       &T->coef[c][lb * 64], 64 * sizeof(uint16_t));
            }

    /* 6. chroma from luma. Per first block, the three sums of
     * src/frontend_quantize.cu:49-74 (x*y, y*y, (b - y)*y over the non-LLF
     * coefficients) in 32 partial FMA chains, chain l over raw positions
     * l, l + 32, ... in order (an LLF position adds fma(0, y, acc)), then an
     * xor-butterfly tree over the 32 partials; the per-tile tree as the
     * reference's. */
    float part[3][64];
    for (int lb = 0; lb < 64; ++lb) {
        float sums3[3] = {0.0f, 0.0f, 0.0f};
        if (bx0 + (lb & 7) < bw && by0 + (lb >> 3) < bh && T->acs[lb] != 0) {
            const int n = T->acs[lb], side = n >> 3;
            float p[3][32];
            for (int l = 0; l < 32; ++l) {
                float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f;
                for (int raw = l; raw < n * n; raw += 32) {
                    const int llf = (raw / n) < side && (raw % n) < side;
                    const int q = raw >> 6;
                    const int idx = (lb + (q / side) * 8 + q % side) * 64 + (raw & 63);
                    const float xr = oracle_h2f(T->coef[0][idx]);
                    const float yr = oracle_h2f(T->coef[1][idx]);
                    const float br = oracle_h2f(T->coef[2][idx]);
                    a0 = fmaf(llf ? 0.0f : xr, yr, a0);
                    a1 = fmaf(llf ? 0.0f : yr, yr, a1);
                    a2 = fmaf(llf ? 0.0f : br - yr, yr, a2);
                }
                p[0][l] = a0; p[1][l] = a1; p[2][l] = a2;
            }
            for (int k = 0; k < 3; ++k) {
                for (int off = 16; off > 0; off >>= 1) {
                    float nx[32];
                    for (int l = 0; l < 32; ++l) nx[l] = p[k][l] + p[k][l ^ off];
                    memcpy(p[k], nx, sizeof(nx));
                }
                sums3[k] = p[k][0];
            }
        }
        part[0][lb] = sums3[0]; part[1][lb] = sums3[1]; part[2][lb] = sums3[2];
    }
    float sums[3];
    for (int k = 0; k < 3; ++k) {
        float v[32];
        for (int l = 0; l < 32; ++l) v[l] = part[k][l] + part[k][l + 32];
        sums[k] = tree32(v);
    }
    int mx, mb;
    oracle_cfl_maps(sums[0], sums[1], sums[2], &mx, &mb);
    out->ytox[ty * cmw + tx] = (int8_t)mx;
    out->ytob[ty * cmw + tx] = (int8_t)mb;

    /* 7. quantisation. */
    const float ytox = (float)mx * (1.0f / 84);
    const float ytob = fmaf((float)mb, 1.0f / 84, 1.0f);
    const size_t cplane = nblocks * 64;
    memset(T->nz, 0, sizeof(T->nz));
    for (int lb = 0; lb < 64; ++lb) {
        const int lbx = lb & 7, lby = lb >> 3;
        if (bx0 + lbx >= bw || by0 + lby >= bh) continue;
        const int f = T->owner[lb], n = T->acs[f], side = n >> 3;
        const int q = (lby - (f >> 3)) * side + lbx - (f & 7);
        const int si = n == 8 ? 0 : (n == 16 ? 1 : 2);
        for (int slot = 0; slot < 64; ++slot) {
            const int raw = q * 64 + slot;
            const size_t g = ((size_t)(by0 + lby) * bw + bx0 + lbx) * 64 + slot;
            int16_t ax = 0, ay = 0, ab = 0;
            if (!((raw / n) < side && (raw % n) < side)) {
                const float qgsf = (float)T->qf[f] * sc->gsf;
                const int k = lb * 64 + slot;
                const float xr = oracle_h2f(T->coef[0][k]);
                const float yr = oracle_h2f(T->coef[1][k]);
                const float br = oracle_h2f(T->coef[2][k]);
                const float wy = g_deq[si][1][raw];
                const int qy = (int)lrintf((yr * qgsf) / wy);
                const float yq = ((float)qy * wy) / qgsf;
                const float wx = g_deq[si][0][raw];
                const int qx = (int)lrintf((fmaf(-ytox, yq, xr) * qgsf) / wx);
                const float wb = g_deq[si][2][raw];
                const int qb = (int)lrintf((fmaf(-ytob, yq, br) * qgsf) / wb);
                ax = (int16_t)qx; ay = (int16_t)qy; ab = (int16_t)qb;
                if (ax) T->nz[0][f]++;
                if (ay) T->nz[1][f]++;
                if (ab) T->nz[2][f]++;
            }
            out->ac[g] = ax;
            out->ac[cplane + g] = ay;
            out->ac[2 * cplane + g] = ab;
        }
    }
    for (int lb = 0; lb < 64; ++lb) {
        if (bx0 + (lb & 7) >= bw || by0 + (lb >> 3) >= bh || T->acs[lb] == 0) continue;
        const int n = T->acs[lb], m = n >> 3;
        const float dcq_x = 4096.0f * sc->dc_scale, dcq_y = 512.0f * sc->dc_scale, dcq_b = 256.0f * sc->dc_scale;
        float llf[3][16], dcv[3][16];
        for (int c = 0; c < 3; ++c)
            for (int fx = 0; fx < m; ++fx)
                for (int fy = 0; fy < m; ++fy) {
                    const int raw = fx * n + fy, q = raw >> 6;
                    llf[c][fx * m + fy] = oracle_h2f(T->coef[c][(lb + (q / m) * 8 + q % m) * 64 + (raw & 63)]);
                }
        for (int c = 0; c < 3; ++c) oracle_dc_from_llf(m, llf[c], dcv[c]);
        for (int oy = 0; oy < m; ++oy)
            for (int ox = 0; ox < m; ++ox) {
                const int p = oy * m + ox;
                const size_t blk = (size_t)(by0 + (lb >> 3) + oy) * bw + bx0 + (lb & 7) + ox;
                const int qdy = (int)lrintf(dcv[1][p] * dcq_y);
                const float ydr = (float)qdy / dcq_y;
                out->dc[nblocks + blk] = qdy;
                out->dc[blk] = (int)lrintf(dcv[0][p] * dcq_x);
                out->dc[2 * nblocks + blk] = (int)lrintf((dcv[2][p] - ydr) * dcq_b);
            }
    }

    /* 8. side information. */
    for (int lb = 0; lb < 64; ++lb) {
        const int gbx = bx0 + (lb & 7), gby = by0 + (lb >> 3);
        if (gbx >= bw || gby >= bh) continue;
        const size_t blk = (size_t)gby * bw + gbx;
        const int f = T->owner[lb], n = T->acs[f];
        const int covered = (n >> 3) * (n >> 3);
        const int l2 = n == 16 ? 2 : (n == 32 ? 4 : 0);
        for (int c = 0; c < 3; ++c) {
            const int nz = T->nz[c][f];
            out->nzn[c * nblocks + blk] = (uint8_t)((nz + covered - 1) >> l2);
            out->nzc[c * nblocks + blk] = (uint16_t)(f == lb ? nz : 0);
        }
        out->acs[blk] = T->acs[lb];
        out->qf[blk] = T->qf[lb];
    }
}

typedef struct {
    const OracleFrame* in;
    const OracleScalars* sc;
    const OracleOutputs* out;
    int ntiles, tw, next;
    pthread_mutex_t mu;
} Work;

static void* worker(void* arg) {
    Work* w = (Work*)arg;
    Tile* T = (Tile*)malloc(sizeof(Tile));
    for (;;) {
        pthread_mutex_lock(&w->mu);
        const int t = w->next++;
        pthread_mutex_unlock(&w->mu);
        if (t >= w->ntiles) break;
        process_tile(w->in, w->sc, w->out, t % w->tw, t / w->tw, T);
    }
    free(T);
    return NULL;
}

int oracle_frontend(const OracleFrame* in, float distance, const OracleOutputs* out, int threads) {
    ensure_tables();
    if (in->width <= 0 || in->height <= 0 || (in->width & 7) || (in->height & 7)) return -1;
    OracleScalars sc;
    oracle_scalars(distance, &sc);
    const int tw = (in->width + 63) / 64, th = (in->height + 63) / 64;
    Work w = {in, &sc, out, tw * th, tw, 0, PTHREAD_MUTEX_INITIALIZER};
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t tids[256];
    for (int i = 0; i < threads; ++i) pthread_create(&tids[i], NULL, worker, &w);
    for (int i = 0; i < threads; ++i) pthread_join(tids[i], NULL);
    return 0;
}

/* Transform selection over a whole plane `y` (width x height, row stride
 * width) with the same costs and decision as the tile path. */
void oracle_select_plane(const float* y, int width, int height, float distance, int8_t* acs) {
    ensure_tables();
    OracleScalars sc;
    oracle_scalars(distance, &sc);
    const int bw = width / 8, bh = height / 8;
    for (int rby = 0; rby < bh; rby += 4)
        for (int rbx = 0; rbx < bw; rbx += 4) {
            float c8[4][4], c16[2][2], c32 = 0.0f;
            for (int dy = 0; dy < 4; ++dy)
                for (int dx = 0; dx < 4; ++dx)
                    if (rbx + dx < bw && rby + dy < bh)
                        c8[dy][dx] = oracle_sel_cost(y + (size_t)(rby + dy) * 8 * width + (rbx + dx) * 8, width, 8,
                                                     sc.qgsf_select);
            for (int qy = 0; qy < 2; ++qy)
                for (int qx = 0; qx < 2; ++qx)
                    if (rbx + 2 * qx + 2 <= bw && rby + 2 * qy + 2 <= bh)
                        c16[qy][qx] = oracle_sel_cost(y + (size_t)(rby + 2 * qy) * 8 * width + (rbx + 2 * qx) * 8,
                                                      width, 16, sc.qgsf_select);
            const int fit32 = rbx + 4 <= bw && rby + 4 <= bh;
            if (fit32) c32 = oracle_sel_cost(y + (size_t)rby * 8 * width + rbx * 8, width, 32, sc.qgsf_select);
            float split = 0.0f;
            int choice[2][2];
            for (int qy = 0; qy < 2; ++qy)
                for (int qx = 0; qx < 2; ++qx) {
                    const int bx = rbx + 2 * qx, by = rby + 2 * qy;
                    float sum8 = 0.0f;
                    int any = 0;
                    for (int dy = 0; dy < 2; ++dy)
                        for (int dx = 0; dx < 2; ++dx)
                            if (bx + dx < bw && by + dy < bh) { sum8 = sum8 + c8[2 * qy + dy][2 * qx + dx]; any = 1; }
                    if (!any) { choice[qy][qx] = -1; continue; }
                    const int fit16 = bx + 2 <= bw && by + 2 <= bh;
                    if (fit16 && c16[qy][qx] <= sum8 + 1.0e-6f) { choice[qy][qx] = 16; split = split + c16[qy][qx]; }
                    else { choice[qy][qx] = 8; split = split + sum8; }
                }
            if (fit32 && c32 <= split + 1.0e-6f) {
                for (int dy = 0; dy < 4; ++dy)
                    for (int dx = 0; dx < 4; ++dx) acs[(rby + dy) * bw + rbx + dx] = (dx == 0 && dy == 0) ? 32 : 0;
                continue;
            }
            for (int qy = 0; qy < 2; ++qy)
                for (int qx = 0; qx < 2; ++qx) {
                    if (choice[qy][qx] < 0) continue;
                    for (int dy = 0; dy < 2; ++dy)
                        for (int dx = 0; dx < 2; ++dx) {
                            const int bx = rbx + 2 * qx + dx, by = rby + 2 * qy + dy;
                            if (choice[qy][qx] == 16) acs[by * bw + bx] = (dx == 0 && dy == 0) ? 16 : 0;
                            else if (bx < bw && by < bh) acs[by * bw + bx] = 8;
                        }
                }
        }
}

/* LLF -> DC resampling of an m x m corner (src/vardct_layout.h:88-111). */
void oracle_dc_from_llf(int m, const float* llf, float* dc) {
    ensure_tables();
    if (m == 1) { dc[0] = llf[0]; return; }
    const double* ob = g_ob[m == 2 ? 0 : 1];
    const double s16[2] = {1.0, 0.901764195028874394};
    const double s32[4] = {1.0, 0.974886821136879522, 0.901764195028874394, 0.787054918159101335};
    const double* scl = m == 2 ? s16 : s32;
    for (int oy = 0; oy < m; ++oy)
        for (int ox = 0; ox < m; ++ox) {
            double sum = 0.0;
            for (int fx = 0; fx < m; ++fx)
                for (int fy = 0; fy < m; ++fy)
                    sum = sum + g_ob[m == 2 ? 0 : 1][fx * 4 + ox] * ob[fy * 4 + oy] * (double)llf[fx * m + fy] * scl[fx] *
                                    scl[fy];
            dc[oy * m + ox] = (float)((double)m * sum);
        }
}

/* CfL regression sums -> map values (src/cfl.h:63-77). */
void oracle_cfl_maps(float sxy, float syy, float sby, int* mx, int* mb) {
    const double dxy = sxy, dyy = syy, dby = sby;
    const float fxr = dyy > 0.0 ? (float)(dxy / dyy) : 0.0f;
    const float fbr = dyy > 0.0 ? (float)(dby / dyy) : 0.0f;
    int x = (int)lrintf(fxr * 84.0f), b = (int)lrintf(fbr * 84.0f);
    *mx = x < -128 ? -128 : (x > 127 ? 127 : x);
    *mb = b < -128 ? -128 : (b > 127 ? 127 : b);
}

/* Individual formulas, exposed for tests. */
float oracle_ratio_gamma(float v, int invert) { ensure_tables(); return ratio_gamma(v, invert); }
float oracle_masking_sqrt(float v) { ensure_tables(); return masking_sqrt(v); }
float oracle_compute_mask(float v) { ensure_tables(); return compute_mask(v); }
void oracle_gaborish_weights(float* out6) { ensure_tables(); memcpy(out6, g_gab, sizeof(g_gab)); }
float oracle_sel_cost(const float* y, int stride, int n, float qgsf) {
    /* Cost of one block whose top-left pixel is y[0] in a plane of row stride `stride`. */
    ensure_tables();
    static __thread float tmp[32 * SS];
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) tmp[r * SS + c] = y[r * stride + c];
    return sel_cost(tmp, 0, 0, n, qgsf);
}
