"""Generates the golden fixtures in tests/golden/ from the reference itself.

Run where the reference tree is present (CUJPEGXL_REFERENCE, else a
"reference" directory beside this repository's root):

    python tests/golden/make_golden.py

Sources of truth, all the reference's own code:
  * oracle/_ref/libjxlref.so, compiled by oracle/build_ref.py from the
    reference's host sources and helper headers: calibration, coefficient
    orders, dequantisation tables, AC context model, Gradient predictor,
    prefix codes, transform selection (decide_region / block_ac_cost),
    LLF -> DC, CfL map quantisation, the XYB pixel formula and AQ helpers
    evaluated with the host libm, and the whole assembly of quantised planes
    into a .jxl file;
  * the reference's tests/reference.py (imported from the reference tree) for
    the centred bilinear chroma upsampling of NV12.
The fixtures are small (.npz / .json); tests compare the CPU restatement and
the CUDA path against them without needing the reference tree.
"""

from __future__ import annotations

import ctypes
import hashlib
import importlib.util
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "tests"))

from oracle import api  # noqa: E402
from oracle import build as obuild  # noqa: E402

import patterns as P  # noqa: E402

REFERENCE = Path(os.environ.get("CUJPEGXL_REFERENCE", REPO.parent / "reference"))


def f32bits(x) -> list[int]:
    return np.asarray(x, np.float32).view(np.uint32).tolist()


def load_reference_py():
    spec = importlib.util.spec_from_file_location("reference_py", REFERENCE / "tests" / "reference.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def huffman_cases(rng: np.random.Generator) -> list[np.ndarray]:
    cases = [np.array([5], np.uint32), np.array([0, 0, 7], np.uint32), np.array([3, 4], np.uint32),
             np.array([1, 1, 1], np.uint32), np.array([1, 2, 3, 4], np.uint32),
             np.array([9, 0, 9, 0, 9, 0, 9], np.uint32), np.array([1, 1, 1, 1, 1], np.uint32)]
    fib = [1, 1]
    while len(fib) < 40:
        fib.append(fib[-1] + fib[-2])
    cases.append(np.array(fib[:30], np.uint32))            # forces the depth limit
    cases.append(np.array(fib[:40][::-1], np.uint32))
    for n in (16, 40, 100, 256):
        for sparsity in (0.0, 0.5, 0.9):
            h = rng.integers(1, 10000, n).astype(np.uint32)
            h[rng.random(n) < sparsity] = 0
            h[-1] = max(h[-1], 1)
            cases.append(h)
    g = np.floor(1e6 * np.exp(-np.arange(200) / 6.0)).astype(np.uint32)
    g[g == 0] = 1
    cases.append(g)
    return cases


def main() -> None:
    obuild.build()
    ref = api.ref()
    rng = np.random.Generator(np.random.PCG64(2024))
    out: dict[str, object] = {}

    # Calibration.
    cal = {}
    for d in (0.05, 0.1, 0.25, 0.5, 0.75, 1.0, 1.5, 2.0, 3.0, 4.0, 6.0, 8.0, 15.0, 25.0):
        ints = np.zeros(3, np.uint32)
        fl = np.zeros(2, np.float32)
        ref.ref_calibrate(d, ints.ctypes.data, fl.ctypes.data)
        cal[repr(d)] = {"global_scale": int(ints[0]), "quant_dc": int(ints[1]), "raw_quant_field": int(ints[2]),
                        "gsf_bits": int(fl.view(np.uint32)[0]), "inv_global_scale_bits": int(fl.view(np.uint32)[1])}
    out["calibration"] = cal

    consts = np.zeros(15, np.float32)
    ref.ref_xyb_constants(consts.ctypes.data)
    gab = np.zeros(6, np.float32)
    ref.ref_gaborish_weights(gab.ctypes.data)
    out["xyb_constants_bits"] = f32bits(consts)
    out["gaborish_weights_bits"] = f32bits(gab)
    (HERE / "constants.json").write_text(json.dumps(out, indent=1, sort_keys=True))

    # Tables and context model.
    tabs = {}
    for n in (8, 16, 32):
        o = np.zeros(n * n, np.uint32)
        ref.ref_natural_order(n, o.ctypes.data)
        tabs[f"order{n}"] = o
        w = np.zeros((3, n * n), np.float32)
        for c in range(3):
            ref.ref_dequant_weights(n, c, w[c].ctypes.data)
        tabs[f"dequant{n}"] = w
    tabs["ac_cluster"] = np.array([ref.ref_ac_cluster(i) for i in range(7425)], np.int32)
    tabs["block_ctx"] = np.array([[ref.ref_ac_block_context(c, o) for o in range(13)] for c in range(3)], np.int32)
    tabs["nonzero_ctx"] = np.array([[ref.ref_ac_nonzero_context(p, b) for b in range(15)] for p in range(80)],
                                   np.uint32)
    zd = []
    for n, cb, l2 in ((8, 1, 0), (16, 4, 2), (32, 16, 4)):
        for left in list(range(1, 70)) + list(range(70, n * n - cb + 1, 7)):
            for k in list(range(cb, min(n * n, cb + 70))) + list(range(cb + 70, n * n, 13)):
                for prev in (0, 1):
                    zd.append((left, k, cb, l2, prev,
                               ref.ref_ac_zero_density_context(left, k, cb, l2, prev)))
    tabs["zero_density"] = np.array(zd, np.uint32)
    gp = []
    for _ in range(4000):
        hl, ht = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        w, n_, nw = (int(v) for v in rng.integers(-3000, 3000, 3))
        gp.append((hl, ht, w, n_, nw, ref.ref_gradient_predict(hl, ht, w, n_, nw)))
    tabs["gradient"] = np.array(gp, np.int64)
    np.savez_compressed(HERE / "tables.npz", **tabs)

    # Prefix codes.
    hz = {}
    for i, h in enumerate(huffman_cases(rng)):
        depth = np.zeros(h.size, np.uint8)
        bits = np.zeros(h.size, np.uint16)
        buf = np.zeros(4096, np.uint8)
        nbits = ref.ref_huffman(h.ctypes.data, h.size, depth.ctypes.data, bits.ctypes.data, buf.ctypes.data,
                                buf.size)
        hz[f"hist{i}"] = h
        hz[f"depth{i}"] = depth
        hz[f"bits{i}"] = bits
        hz[f"header{i}"] = buf[: (nbits + 7) // 8]
        hz[f"nbits{i}"] = np.array([nbits], np.int64)
    np.savez_compressed(HERE / "huffman.npz", **hz)

    # XYB formula on exact bilinear chroma (reference tests/reference.py).
    refpy = load_reference_py()
    w, h = 96, 64
    from cujpegxl_b200.synth import make_nv12

    nv = make_nv12(w, h, 9)
    chroma = nv[w * h:].reshape(h // 2, w).astype(np.float64)
    cb = refpy.upsample_chroma(chroma[:, 0::2], w, h) / 255.0
    cr = refpy.upsample_chroma(chroma[:, 1::2], w, h) / 255.0
    yv = nv[: w * h].reshape(h, w).astype(np.float32) * np.float32(1.0 / 255.0)
    xyb = np.zeros((3, h, w), np.float32)
    x, y_, b = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    for yy in range(h):
        for xx in range(w):
            ref.ref_xyb_pixel(float(yv[yy, xx]), float(np.float32(cb[yy, xx])), float(np.float32(cr[yy, xx])),
                              ctypes.byref(x), ctypes.byref(y_), ctypes.byref(b))
            xyb[:, yy, xx] = (x.value, y_.value, b.value)
    srgb = refpy.nv12_to_srgb(nv.tobytes(), w, h)
    np.savez_compressed(HERE / "xyb.npz", nv12=nv, width=w, height=h, xyb=xyb, srgb=srgb,
                        cb=cb.astype(np.float32), cr=cr.astype(np.float32))

    # AQ helpers (reference formulas with the host libm).
    v = np.concatenate([np.linspace(-0.1, 1.5, 401), np.linspace(0.0, 0.25, 101)]).astype(np.float32)
    mv = np.linspace(0.0, 8.0, 301).astype(np.float32)
    np.savez_compressed(
        HERE / "aq_helpers.npz", v=v, mv=mv,
        ratio_true=np.array([ref.ref_ratio_cbrt_gamma(float(t), 1) for t in v], np.float32),
        ratio_false=np.array([ref.ref_ratio_cbrt_gamma(float(t), 0) for t in v], np.float32),
        masking_sqrt=np.array([ref.ref_masking_sqrt(float(t)) for t in np.clip(v, 0, None)], np.float32),
        compute_mask=np.array([ref.ref_compute_mask(float(t)) for t in mv], np.float32))

    # Transform selection on a sharpened plane (decide_region), and block costs.
    sw, sh = 136, 96
    fr = api.frontend(make_nv12(sw, sh, 4), sw, sh, 1.0, debug=True)
    yplane = fr.sharp[sw * sh: 2 * sw * sh].copy()
    sel = {"y": yplane, "width": sw, "height": sh}
    for d in (0.5, 1.0, 2.0, 4.0):
        sel[f"acs_{d}"] = api.ref_select(yplane, sw, sh, d)
    costs = []
    for (px, py, n) in ((0, 0, 8), (8, 16, 8), (64, 32, 8), (16, 16, 16), (96, 64, 16), (0, 0, 32), (64, 32, 32)):
        for d in (0.5, 1.0, 2.0):
            qg = api.scalars(d)["qgsf_select"]
            c = ref.ref_block_ac_cost(yplane.ctypes.data, sw, px, py, n, qg)
            costs.append((px, py, n, np.float32(qg).view(np.uint32), np.float32(c).view(np.uint32)))
    sel["costs"] = np.array(costs, np.uint64)
    np.savez_compressed(HERE / "selection.npz", **sel)

    # LLF -> DC and CfL maps.
    llf = {}
    for m in (2, 4):
        ins = rng.normal(0, 0.3, (50, m * m)).astype(np.float32)
        outs = np.zeros_like(ins)
        for i in range(ins.shape[0]):
            ref.ref_dc_from_llf(m, ins[i].ctypes.data, outs[i].ctypes.data)
        llf[f"in{m}"] = ins
        llf[f"out{m}"] = outs
    sums = rng.normal(0, 1, (500, 3)).astype(np.float32)
    sums[:, 1] = np.abs(sums[:, 1]) * rng.choice([0.0, 1e-6, 1.0, 100.0], 500).astype(np.float32)
    mx = ctypes.c_int()
    mb = ctypes.c_int()
    maps = []
    for s in sums:
        ref.ref_cfl_maps_from_sums(float(s[0]), float(s[1]), float(s[2]), ctypes.byref(mx), ctypes.byref(mb))
        maps.append((mx.value, mb.value))
    llf["cfl_sums"] = sums
    llf["cfl_maps"] = np.array(maps, np.int32)
    np.savez_compressed(HERE / "llf_cfl.npz", **llf)

    # Whole-file assembly of quantised planes by the reference's host pieces.
    files = {}
    cases = {"dct8_512x384": (P.empty(512, 384), 4096, 32), "mixed_512x384": (P.mixed_full(512, 384), 4096, 32),
             "mixed_qf_264x264": (P.mixed_full(264, 264, seed=5), 9502, 61),
             "mixed_2560x2304": (P.mixed_full(2560, 2304), 4096, 32)}
    P.fill_ac_pattern(cases["dct8_512x384"][0])
    P.fill_dc_pattern(cases["dct8_512x384"][0])
    for name, (f, gs, qdc) in cases.items():
        r = api.FrontendResult(f["w"], f["h"])
        for k, vv in P.flat(f).items():
            getattr(r, k)[...] = vv
        ac32 = r.ac.astype(np.int32)
        buf = np.zeros(3 * r.acs.size * 384 + (1 << 20), np.uint8)
        nbytes = ref.ref_encode_frame(f["w"], f["h"], ac32.ctypes.data, r.dc.ctypes.data, r.acs.ctypes.data,
                                      r.ytox.ctypes.data, r.ytob.ctypes.data, r.qf.ctypes.data, gs, qdc,
                                      buf.ctypes.data, buf.size)
        data = buf[:nbytes]
        files[name] = {"global_scale": gs, "quant_dc": qdc, "size": int(nbytes),
                       "sha256": hashlib.sha256(data.tobytes()).hexdigest()}
        if nbytes < 200_000:
            np.save(HERE / f"file_{name}.npy", data)
    (HERE / "files.json").write_text(json.dumps(files, indent=1, sort_keys=True))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
