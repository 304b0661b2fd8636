"""The float stages that the reference runs only on its device, pinned by
evaluating the reference's own formulas here, independently of the CPU
restatement's code:

* inverse gaborish: the 5x5 stencil of src/frontend_transform.cu:19-36 with
  the weights of src/gaborish.h:16-28, evaluated in float64 on the
  restatement's XYB planes, against the restatement's sharpened planes;
* the adaptive quant field: src/frontend_fused.cu:54-204 and
  src/adaptive_quant_impl.cuh:30-116 (32x32-pixel tiles, pre-erosion cells of
  4x4 pixels, FuzzyErosion clamped to the tile, HF/gamma/blue modulations,
  exp tail) in float64 on the same XYB planes, against the quant field;
* the quantiser: src/frontend_quantize.cu:125-201 restated in numpy float32
  on the restatement's own FP16 coefficients must give its integers exactly
  (the exact-rint check of tests/quant_selfconsistency_test.py:126-179), and
  every AC and DC value must reconstruct within half a quantisation step (the
  bound of src/frontend_quantize_gpu_test.cc:142-246);
* the CfL maps: the per-block sums in the reference's single chain per block
  (src/frontend_quantize.cu:49-74) and its 64-entry tile tree, quantised as
  src/cfl.h:58-77, against the maps of the restatement's 32-chain warp sums;
  equal except next to a rounding boundary.

The CUDA path equals the restatement bit for bit (tests/test_gpu_parity.py),
so these pins hold for it too.
"""

from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np
import pytest

from cujpegxl_b200.synth import make_nv12
from oracle import api

from . import patterns as P

GOLD = Path(__file__).resolve().parent / "golden"

CASES = [(264, 264, 1.0, 11), (520, 392, 2.0, 4), (384, 320, 0.5, 7)]


@pytest.fixture(scope="module", params=CASES, ids=lambda c: f"{c[0]}x{c[1]}-d{c[2]}")
def frame(request):
    w, h, d, seed = request.param
    r = api.frontend(make_nv12(w, h, seed), w, h, d, debug=True)
    return w, h, d, r


def _clamped(plane: np.ndarray, pad: int) -> np.ndarray:
    return np.pad(plane, pad, mode="edge")


# ---- inverse gaborish -------------------------------------------------------------

def test_gaborish_plane_matches_reference_stencil(frame):
    """Every sharpened sample within 1e-5 of the stencil's magnitude
    sum(|w_i p_i|) of the float64 value (the relative bound of a float sum
    of those terms), and within 1e-5 relative where it is not cancelled."""
    w, h, d, r = frame
    wc, wr, wr2, wd, wl, wd2 = np.array(json.loads((GOLD / "constants.json").read_text())[
        "gaborish_weights_bits"], np.uint32).view(np.float32).astype(np.float64)
    taps = [((0, 0), wc)]
    taps += [((dx, dy), wr) for dx, dy in ((-1, 0), (1, 0), (0, -1), (0, 1))]
    taps += [((dx, dy), wr2) for dx, dy in ((-2, 0), (2, 0), (0, -2), (0, 2))]
    taps += [((dx, dy), wd) for dx, dy in ((-1, -1), (1, -1), (-1, 1), (1, 1))]
    taps += [((dx, dy), wl) for dx, dy in ((-2, -1), (2, -1), (-2, 1), (2, 1), (-1, -2), (1, -2), (-1, 2), (1, 2))]
    taps += [((dx, dy), wd2) for dx, dy in ((-2, -2), (2, -2), (-2, 2), (2, 2))]
    xyb = r.xyb.reshape(3, h, w).astype(np.float64)
    got = r.sharp.reshape(3, h, w).astype(np.float64)
    for c in range(3):
        p = _clamped(xyb[c], 2)
        want = np.zeros((h, w))
        mag = np.zeros((h, w))
        for (dx, dy), wt in taps:
            t = wt * p[2 + dy:2 + dy + h, 2 + dx:2 + dx + w]
            want += t
            mag += np.abs(t)
        err = np.abs(got[c] - want)
        assert np.all(err <= 1e-5 * mag), (c, float((err / mag).max()))
        big = np.abs(want) > 0.1 * mag
        assert np.all(err[big] <= 1e-5 * np.abs(want[big])), c


# ---- adaptive quant field ------------------------------------------------------------

# src/adaptive_quant_impl.cuh:16-27 and src/frontend_fused.cu:139-196 (libjxl's
# AdaptiveQuantizationMap constants).
K_SG_MUL = 226.77216153508914
K_SG_MUL2 = 1.0 / 73.377132366608819
K_SG_LOG2 = 0.693147181
K_SG_RET_MUL = K_SG_MUL2 * 18.6580932135 * K_SG_LOG2
K_SG_V_OFFSET = 7.7825991679894591
K_AC_QUANT = 0.725          # src/quant_calibration.h:30
K_QUANT_MAX = 256           # src/quant_calibration.h:37


def ratio_cbrt_gamma(v: np.ndarray, invert: bool) -> np.ndarray:
    eps = 1e-2
    v = np.maximum(v, 0.0)
    num = K_SG_RET_MUL * 3.0 * K_SG_MUL * v * v + eps
    den = K_SG_LOG2 * K_SG_MUL * v * v * v + (K_SG_V_OFFSET * K_SG_LOG2 + eps)
    return num / den if invert else den / num


def masking_sqrt(v: np.ndarray) -> np.ndarray:
    return 0.25 * np.sqrt(v * math.sqrt(211.66567973503678 * 1e8) + 27.505837037000106)


def compute_mask(out_val: np.ndarray) -> np.ndarray:
    k_offset3 = 3.7179635626140772
    v1 = np.maximum(out_val * 0.80061762862741759, 1e-3)
    v2 = 1.0 / (v1 + 302.59587815579727)
    v3 = 1.0 / (v1 * v1 + k_offset3)
    v4 = 1.0 / (v1 * v1 + 0.25 * k_offset3)
    return -0.7647 + 9.4708735624378946 * v4 + 17.35036561631863 * v2 + 6.7943250517376494 * v3


def aq_params(distance: float) -> tuple[float, float, list[float]]:
    """mul_pb, add_pb and the FuzzyErosion weights (src/frontend_fused.cu:215-239)."""
    scale = K_AC_QUANT / distance
    dampen = 1.0
    if distance >= 2.0:
        dampen = max(0.0, 1.0 - (distance - 2.0) / 12.0)
    mul_pb = scale * dampen
    add_pb = (1.0 - dampen) * 0.48 * scale
    efm = (2.0 - distance) * 0.5 if distance < 2.0 else 0.0
    km = [0.125, 0.10 - efm * 0.10, 0.09 - efm * 0.09, 0.06 - efm * 0.06]
    norm = 0.29959705784054957 / sum(km)
    return mul_pb, add_pb, [k * norm for k in km]


def reference_quant_field(xyb: np.ndarray, w: int, h: int, distance: float, inv_gs: float) -> np.ndarray:
    """The fused AQ kernel's quant field in float64: returns the value before
    truncation, qval * inv_global_scale + 0.5, per block."""
    mul_pb, add_pb, km = aq_params(distance)
    bw, bh = w // 8, h // 8
    tx, ty = (bw + 3) // 4, (bh + 3) // 4
    X, Y, B = (xyb[c] for c in range(3))
    # Pre-erosion cells over every pixel of every (possibly partial) tile: the
    # tile loads clamped coordinates, so pixels past the frame repeat its edge.
    Hp, Wp = ty * 32, tx * 32
    Yp = _clamped(Y, 1)
    Yp = np.pad(Yp, ((0, Hp + 2 - Yp.shape[0]), (0, Wp + 2 - Yp.shape[1])), mode="edge") if (
        Hp + 2 > Yp.shape[0] or Wp + 2 > Yp.shape[1]) else Yp
    c = Yp[1:Hp + 1, 1:Wp + 1]
    base = 0.25 * (Yp[2:Hp + 2, 1:Wp + 1] + Yp[0:Hp, 1:Wp + 1] + Yp[1:Hp + 1, 0:Wp] + Yp[1:Hp + 1, 2:Wp + 2])
    diff = ratio_cbrt_gamma(c + 0.019, False) * (c - base)
    diff = np.minimum(diff * diff, 0.2)
    pre = 0.25 * masking_sqrt(diff).reshape(Hp // 4, 4, Wp // 4, 4).sum(axis=(1, 3))  # [cy][cx]
    # FuzzyErosion per 32x32 tile (8x8 cells), neighbourhood clamped to the tile.
    er_cells = np.zeros_like(pre)
    for cy in range(Hp // 4):
        for cx in range(Wp // 4):
            t0y, t0x = (cy // 8) * 8, (cx // 8) * 8
            ly, lx = cy - t0y, cx - t0x
            ys = [min(max(ly + k, 0), 7) + t0y for k in (-1, 0, 1)]
            xs = [min(max(lx + k, 0), 7) + t0x for k in (-1, 0, 1)]
            nb = sorted(pre[yy, xx] for yy in ys for xx in xs)[:4]
            # With repeated neighbours at the clamp the kernel's insertion
            # keeps duplicates, as a sort of the nine values with repeats does.
            er_cells[cy, cx] = km[0] * nb[0] + km[1] * nb[1] + km[2] * nb[2] + km[3] * nb[3]
    aq = er_cells.reshape(Hp // 8, 2, Wp // 8, 2).sum(axis=(1, 3))[:bh, :bw]
    # Per-block modulation sums over the 8x8 pixels (frame planes, no halo).
    Yb = Y[:bh * 8, :bw * 8].reshape(bh, 8, bw, 8)
    Xb = X[:bh * 8, :bw * 8].reshape(bh, 8, bw, 8)
    Bb = B[:bh * 8, :bw * 8].reshape(bh, 8, bw, 8)
    hf = np.minimum(0.0206, np.abs(Yb[:, :, :, :7] - Yb[:, :, :, 1:])).sum(axis=(1, 3))
    hf += np.minimum(0.0206, np.abs(Yb[:, :7] - Yb[:, 1:])).sum(axis=(1, 3))
    iny = Yb + 0.16
    gamma = (ratio_cbrt_gamma(iny - Xb, True) + ratio_cbrt_gamma(iny + Xb, True)).sum(axis=(1, 3)) * (0.5 / 64.0)
    k_limit = 0.027121074570634722
    pye = Yb + 0.084381641171960495 + np.abs(Xb)
    blue = np.where(Bb > pye, np.minimum(Bb - pye, k_limit), 0.0).sum(axis=(1, 3))
    blue = np.where(blue >= 32.0 * k_limit, 64.0 * k_limit - blue, blue)
    blue = np.minimum(blue, 15.398788439047934 * k_limit)
    ov = compute_mask(aq) + hf * -0.38 + 0.42 + 0.1005613337192697 * np.log2(gamma) + blue * 0.14207000358439159
    qval = np.exp(ov) * mul_pb + add_pb
    return qval * inv_gs + 0.5


def test_quant_field_matches_reference_formula(frame):
    """qf equals the float64 evaluation's truncation, clamped to [1, 256],
    wherever that value lies more than 1e-4 relative from an integer; the
    blocks within that band are counted and must be rare."""
    w, h, d, r = frame
    cal = json.loads((GOLD / "constants.json").read_text())["calibration"][str(d)]
    inv_gs = float(np.uint32(cal["inv_global_scale_bits"]).view(np.float32))
    xyb = r.xyb.reshape(3, h, w).astype(np.float64)
    v = reference_quant_field(xyb, w, h, d, inv_gs)
    want = np.clip(np.floor(v), 1, K_QUANT_MAX).astype(np.int64).ravel()
    got = r.qf.astype(np.int64)
    near = np.abs(v - np.rint(v)).ravel() <= 1e-4 * np.abs(v).ravel()
    bad = (got != want) & ~near
    assert not bad.any(), (int(bad.sum()), np.flatnonzero(bad)[:8].tolist())
    assert np.all(np.abs(got - want) <= 1)
    assert near.mean() < 0.01, float(near.mean())
    assert len(np.unique(got)) > 4, "the field must vary across the frame"


# ---- quantiser ------------------------------------------------------------------------

def _f32(x) -> np.ndarray:
    return np.asarray(x, np.float32)


def _fma32(a, b, c) -> np.ndarray:
    """Single-rounding float32 a*b + c (the product is exact in long double)."""
    ld = np.longdouble
    return (a.astype(ld) * b.astype(ld) + c.astype(ld)).astype(np.float32)


def _dequant(n: int) -> np.ndarray:
    return np.load(GOLD / "tables.npz")[f"dequant{n}"]


def test_quantiser_exact_rint_and_half_step(frame):
    w, h, d, r = frame
    s = api.scalars(d)
    gsf = np.float32(s["gsf"])
    dc_scale = np.float32(s["dc_scale"])
    bw, bh = w // 8, h // 8
    nb = bw * bh
    cmw = (bw + 7) // 8
    coef = r.coeff.view(np.float16).astype(np.float32)
    ac = r.ac.astype(np.int64)
    acs = r.acs.reshape(bh, bw)
    checked = 0
    for by in range(bh):
        for bx in range(bw):
            n = int(acs[by, bx])
            if n == 0:
                continue
            m = n // 8
            tile = (by // 8) * cmw + bx // 8
            # cfl_ytox_ratio / cfl_ytob_ratio (src/cfl.h:36-41): base + m / 84,
            # the B form contracted to one FMA as the device compiles it.
            ytox = np.float32(np.float32(int(r.ytox[tile])) * np.float32(1.0 / 84))
            ytob = _fma32(_f32([int(r.ytob[tile])]), _f32([1.0 / 84]), _f32([1.0]))[0]
            qgsf = np.float32(np.float32(int(r.qf[by * bw + bx])) * gsf)
            raws = np.array([raw for raw in range(n * n) if not (raw // n < m and raw % n < m)])
            slots = np.array([P.covered_slot(n, bx, by, bw, int(raw)) for raw in raws])
            wx, wy, wb = (_dequant(n)[c][raws] for c in range(3))
            xr, yr, br = (coef[c * nb * 64 + slots] for c in range(3))
            qy = np.rint(_f32(_f32(yr * qgsf) / wy))
            yq = _f32(_f32(qy.astype(np.float32) * wy) / qgsf)
            qx = np.rint(_f32(_f32(_fma32(np.full_like(yq, -ytox), yq, xr) * qgsf) / wx))
            qb = np.rint(_f32(_f32(_fma32(np.full_like(yq, -ytob), yq, br) * qgsf) / wb))
            np.testing.assert_array_equal(ac[nb * 64 + slots], qy, err_msg=f"Y at {bx},{by}")
            np.testing.assert_array_equal(ac[slots], qx, err_msg=f"X at {bx},{by}")
            np.testing.assert_array_equal(ac[2 * nb * 64 + slots], qb, err_msg=f"B at {bx},{by}")
            # Half-step reconstruction with CfL inverted (frontend_quantize_gpu_test.cc:205-212).
            y_round = ac[nb * 64 + slots] * wy.astype(np.float64) / qgsf
            x_rec = ac[slots] * wx.astype(np.float64) / qgsf + float(ytox) * y_round
            b_rec = ac[2 * nb * 64 + slots] * wb.astype(np.float64) / qgsf + float(ytob) * y_round
            assert np.all(np.abs(x_rec - xr) <= 0.5 * wx / qgsf + 1e-4)
            assert np.all(np.abs(b_rec - br) <= 0.5 * wb / qgsf + 1e-4)
            assert np.all(np.abs(y_round - yr) <= 0.5 * wy / qgsf + 1e-4)
            checked += raws.size
            # DC: dequantised values within half a DC step of the LLF -> DC
            # resampling of the stored coefficients, Y removed from B
            # (frontend_quantize_gpu_test.cc:214-239).
            llf = np.zeros((3, m * m), np.float32)
            for c in range(3):
                for fx in range(m):
                    for fy in range(m):
                        llf[c, fx * m + fy] = coef[c * nb * 64 + P.covered_slot(n, bx, by, bw, fx * n + fy)]
            dcv = np.zeros((3, m * m), np.float32)
            for c in range(3):
                if m == 1:
                    dcv[c] = llf[c]
                else:
                    api.oracle().oracle_dc_from_llf(m, np.ascontiguousarray(llf[c]).ctypes.data,
                                                    dcv[c].ctypes.data)
            q = [4096.0 * float(dc_scale), 512.0 * float(dc_scale), 256.0 * float(dc_scale)]
            for oy in range(m):
                for ox in range(m):
                    p = oy * m + ox
                    blk = (by + oy) * bw + bx + ox
                    y_dc = r.dc[nb + blk] / q[1]
                    assert abs(y_dc - dcv[1, p]) <= 0.5 / q[1] + 1e-3
                    assert abs(r.dc[blk] / q[0] - dcv[0, p]) <= 0.5 / q[0] + 1e-3
                    assert abs(r.dc[2 * nb + blk] / q[2] + y_dc - dcv[2, p]) <= 0.5 / q[2] + 1e-3
    assert checked > 1000


# ---- chroma-from-luma maps --------------------------------------------------------------

def _ref_order_sums(coef: np.ndarray, acs: np.ndarray, bw: int, bh: int) -> np.ndarray:
    """The reference's per-block sums (src/frontend_quantize.cu:49-74): one
    chain per first block over its non-LLF coefficients in raw order, FMA
    products of the FP16 values; [3][bh][bw] (zero off first blocks)."""
    ld = np.longdouble
    nb = bw * bh
    out = np.zeros((3, bh, bw), np.float32)
    for n in (8, 16, 32):
        ys, xs = np.nonzero(acs == n)
        if ys.size == 0:
            continue
        side = n // 8
        acc = np.zeros((3, ys.size), np.float32)
        for raw in range(n * n):
            if raw // n < side and raw % n < side:
                continue
            q = raw // 64
            slots = ((ys + q // side) * bw + xs + q % side) * 64 + raw % 64
            x, y, b = (coef[c * nb * 64 + slots].astype(np.float32) for c in range(3))
            acc[0] = (x.astype(ld) * y + acc[0]).astype(np.float32)
            acc[1] = (y.astype(ld) * y + acc[1]).astype(np.float32)
            acc[2] = ((b - y).astype(np.float32).astype(ld) * y + acc[2]).astype(np.float32)
        out[:, ys, xs] = acc
    return out


def test_cfl_maps_match_reference_order(frame):
    """The CfL sums run as 32 interleaved partial chains and a tree across a
    warp; the maps must equal those of the reference's single chain per block
    (and its 64-entry tile tree) except where the quotient times 84 lies
    within 1e-4 (relative) of a rounding boundary."""
    w, h, d, r = frame
    bw, bh = w // 8, h // 8
    cmw = (bw + 7) // 8
    coef = r.coeff.view(np.float16)
    part = _ref_order_sums(coef, r.acs.reshape(bh, bw), bw, bh)
    near = checked = 0
    for ty in range((bh + 7) // 8):
        for tx in range(cmw):
            p = np.zeros((3, 64), np.float32)
            sub = part[:, ty * 8:ty * 8 + 8, tx * 8:tx * 8 + 8]
            for c in range(3):
                blk = np.zeros((8, 8), np.float32)
                blk[:sub.shape[1], :sub.shape[2]] = sub[c]
                v = blk.ravel()
                s = 32
                while s > 0:
                    v = v.copy()
                    v[:s] = v[:s] + v[s:2 * s]
                    s //= 2
                p[c, 0] = v[0]
            sxy, syy, sby = (float(p[c, 0]) for c in range(3))
            want = []
            for num in (sxy, sby):
                f = np.float32(num / syy) if syy > 0 else np.float32(0.0)
                v84 = float(np.float32(f * np.float32(84.0)))
                want.append((int(np.clip(np.rint(v84), -128, 127)), v84))
            got = (int(r.ytox[ty * cmw + tx]), int(r.ytob[ty * cmw + tx]))
            for (m, v84), g in zip(want, got):
                checked += 1
                if m != g:
                    assert abs(abs(v84 - np.floor(v84)) - 0.5) <= 1e-4 * max(1.0, abs(v84)), (tx, ty, m, g, v84)
                    near += 1
    assert checked > 20 and near <= max(1, checked // 100)
