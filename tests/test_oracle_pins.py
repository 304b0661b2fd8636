"""The CPU restatement pinned against the reference: golden fixtures made by
tests/golden/make_golden.py from the reference's own code, plus live
comparisons with the reference-built checker (oracle/_ref) when it is present.
Integer and bitstream results are exact; float formulas evaluated with a
different libm are held to a few ulp.
"""

from __future__ import annotations

import ctypes
import json
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import api

from . import patterns as P

GOLD = Path(__file__).resolve().parent / "golden"
REPO = GOLD.parents[1]


def ulps(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    ai = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    bi = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    ai = np.where(ai < 0, -(ai & 0x7FFFFFFF), ai)
    bi = np.where(bi < 0, -(bi & 0x7FFFFFFF), bi)
    return np.abs(ai - bi)


def test_calibration_exact():
    gold = json.loads((GOLD / "constants.json").read_text())["calibration"]
    for d, g in gold.items():
        s = api.scalars(float(d))
        assert (s["global_scale"], s["quant_dc"], s["raw_quant_field"]) == (
            g["global_scale"], g["quant_dc"], g["raw_quant_field"]), d
        assert np.float32(s["gsf"]).view(np.uint32) == g["gsf_bits"]
        assert np.float32(s["inv_global_scale"]).view(np.uint32) == g["inv_global_scale_bits"]


def test_gaborish_weights_exact():
    gold = json.loads((GOLD / "constants.json").read_text())["gaborish_weights_bits"]
    w = np.zeros(6, np.float32)
    api.oracle().oracle_gaborish_weights(w.ctypes.data)
    assert w.view(np.uint32).tolist() == gold


def test_product_constants_match_reference_values():
    """The product's constants header carries the reference's values."""
    gold = json.loads((GOLD / "constants.json").read_text())["xyb_constants_bits"]
    src = (REPO / "cujpegxl_b200" / "csrc" / "jxl_constants.cuh").read_text()
    names = ["kM00", "kM01", "kM02", "kM10", "kM11", "kM12", "kM20", "kM21", "kM22", "kOpsinBias",
             "kCrToR", "kCbToG", "kCrToG", "kCbToB", "kChromaCenter"]
    env = {}
    # Evaluate the simple `a op b op c` definitions in file order, left to
    # right in float32 as the compiler folds them.
    for name, expr in re.findall(r"constexpr float (kM[0-2][0-2]|kOpsinBias|kCrTo\w+|kCbTo\w+|kChromaCenter) = ([^;]+);",
                                 src):
        toks = re.split(r"\s*([-+*/])\s*", expr.strip())

        def val(t: str) -> np.float32:
            return env[t] if t in env else np.float32(float(t.rstrip("f")))

        acc = val(toks[0])
        for op, t in zip(toks[1::2], toks[2::2]):
            v = val(t)
            acc = {"+": acc + v, "-": acc - v, "*": acc * v, "/": acc / v}[op]
        env[name] = np.float32(acc)
    got = [int(np.float32(env[n]).view(np.uint32)) for n in names]
    assert got == gold


def test_dequant_tables_match_reference():
    t = np.load(GOLD / "tables.npz")
    text = (REPO / "cujpegxl_b200" / "csrc" / "jxl_dequant_tables.inc").read_text()
    for n in (8, 16, 32):
        block = text.split(f"kDequantBits{n}[3][{n * n}] = {{", 1)[1].split("};", 1)[0]
        words = np.array([int(w, 16) for w in re.findall(r"0x([0-9a-f]{8})u", block)], np.uint32)
        np.testing.assert_array_equal(words.view(np.float32).reshape(3, n * n), t[f"dequant{n}"])


def test_huffman_exact():
    z = np.load(GOLD / "huffman.npz")
    i = 0
    while f"hist{i}" in z:
        h = z[f"hist{i}"].astype(np.uint32)
        depth = np.zeros(h.size, np.uint8)
        bits = np.zeros(h.size, np.uint16)
        buf = np.zeros(4096, np.uint8)
        nbits = api.oracle().oracle_huffman(h.ctypes.data, h.size, depth.ctypes.data, bits.ctypes.data,
                                            buf.ctypes.data, buf.size)
        assert nbits == int(z[f"nbits{i}"][0]), i
        np.testing.assert_array_equal(depth, z[f"depth{i}"], err_msg=f"case {i}")
        np.testing.assert_array_equal(bits, z[f"bits{i}"], err_msg=f"case {i}")
        np.testing.assert_array_equal(buf[: (nbits + 7) // 8], z[f"header{i}"], err_msg=f"case {i}")
        i += 1
    assert i > 20


def test_xyb_formula_within_tolerance():
    """XYB of exact-bilinear NV12 pixels vs the reference's formula with the
    host libm: within 1e-5 relative (plus 1e-7 absolute near zero)."""
    z = np.load(GOLD / "xyb.npz")
    w, h = int(z["width"]), int(z["height"])
    nv = z["nv12"]
    luma = nv[: w * h]
    chroma = nv[w * h:]
    fr = api._Frame(luma.ctypes.data, chroma.ctypes.data, w, w, w, h)
    got = np.zeros((3, h, w), np.float32)
    o3 = np.zeros(3, np.float32)
    for y in range(h):
        for x in range(w):
            api.oracle().oracle_xyb_pixel(ctypes.byref(fr), x, y, o3.ctypes.data)
            got[:, y, x] = o3
    want = z["xyb"]
    err = np.abs(got.astype(np.float64) - want)
    assert np.all(err <= 1e-5 * np.abs(want) + 1e-7), err.max()


def test_aq_helpers_within_tolerance():
    z = np.load(GOLD / "aq_helpers.npz")
    o = api.oracle()
    for v, t, f in zip(z["v"], z["ratio_true"], z["ratio_false"]):
        assert ulps(o.oracle_ratio_gamma(float(v), 1), t) <= 4
        assert ulps(o.oracle_ratio_gamma(float(v), 0), f) <= 4
    for v, m in zip(np.clip(z["v"], 0, None), z["masking_sqrt"]):
        assert ulps(o.oracle_masking_sqrt(float(v)), m) <= 4
    for v, m in zip(z["mv"], z["compute_mask"]):
        assert abs(o.oracle_compute_mask(float(v)) - m) <= 4e-7 * max(1.0, abs(float(m)))


def test_selection_exact():
    z = np.load(GOLD / "selection.npz")
    w, h = int(z["width"]), int(z["height"])
    y = z["y"].astype(np.float32)
    for d in (0.5, 1.0, 2.0, 4.0):
        acs = np.full((w // 8) * (h // 8), -1, np.int8)
        api.oracle().oracle_select_plane(y.ctypes.data, w, h, d, acs.ctypes.data)
        np.testing.assert_array_equal(acs, z[f"acs_{d}"], err_msg=f"d={d}")
    for px, py, n, qg_bits, cost_bits in z["costs"]:
        qg = np.uint32(qg_bits).view(np.float32)
        sub = y[int(py) * w + int(px):]
        c = api.oracle().oracle_sel_cost(sub.ctypes.data, w, int(n), float(qg))
        assert np.float32(c).view(np.uint32) == np.uint32(cost_bits), (px, py, n)


def test_llf_dc_and_cfl_exact():
    z = np.load(GOLD / "llf_cfl.npz")
    for m in (2, 4):
        for a, b in zip(z[f"in{m}"], z[f"out{m}"]):
            a = np.ascontiguousarray(a)
            out = np.zeros(m * m, np.float32)
            api.oracle().oracle_dc_from_llf(m, a.ctypes.data, out.ctypes.data)
            np.testing.assert_array_equal(out.view(np.uint32), b.view(np.uint32))
    mx, mb = ctypes.c_int(), ctypes.c_int()
    for s, m in zip(z["cfl_sums"], z["cfl_maps"]):
        api.oracle().oracle_cfl_maps(ctypes.c_float(s[0]), ctypes.c_float(s[1]), ctypes.c_float(s[2]),
                                     ctypes.byref(mx), ctypes.byref(mb))
        assert (mx.value, mb.value) == tuple(m)


def _oracle_file(f: dict, gs: int, qdc: int) -> bytes:
    r = api.FrontendResult(f["w"], f["h"])
    for k, v in P.flat(f).items():
        getattr(r, k)[...] = v
    cap = 3 * r.acs.size * 384 + (1 << 20)
    out = np.zeros(cap, np.uint8)
    n = api.oracle().oracle_assemble(f["w"], f["h"], r.ac.ctypes.data, r.dc.ctypes.data, r.acs.ctypes.data,
                                     r.qf.ctypes.data, r.ytox.ctypes.data, r.ytob.ctypes.data, gs, qdc,
                                     out.ctypes.data, cap)
    return out[:n].tobytes()


@pytest.mark.parametrize("name", ["dct8_512x384", "mixed_512x384", "mixed_qf_264x264", "mixed_2560x2304"])
def test_assembly_matches_reference_files(name):
    import hashlib

    meta = json.loads((GOLD / "files.json").read_text())[name]
    w, h = (int(v) for v in name.rsplit("_", 1)[1].split("x"))
    if name.startswith("dct8"):
        f = P.empty(w, h)
        P.fill_ac_pattern(f)
        P.fill_dc_pattern(f)
    else:
        f = P.mixed_full(w, h, seed=5 if "qf" in name else None)
    data = _oracle_file(f, meta["global_scale"], meta["quant_dc"])
    assert len(data) == meta["size"]
    assert hashlib.sha256(data).hexdigest() == meta["sha256"]


@pytest.mark.skipif(not api.ref_available(), reason="reference-built checker not present")
def test_frontend_then_assembly_matches_reference_live():
    """Synthetic frame: the restatement's planes assembled by the reference's
    host pieces give the same file as the restatement's own assembly, and its
    transform decisions equal decide_region's on its sharpened plane."""
    from cujpegxl_b200.synth import make_nv12

    for (w, h, d, seed) in ((520, 392, 1.0, 1), (264, 264, 2.0, 2)):
        nv = make_nv12(w, h, seed)
        r = api.frontend(nv, w, h, d, debug=True)
        assert api.assemble(r, d) == api.ref_encode_frame(r, d)
        np.testing.assert_array_equal(api.ref_select(r.sharp[w * h: 2 * w * h], w, h, d), r.acs)
