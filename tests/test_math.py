"""The deterministic transcendentals and FP16 conversions of the restatement
(the CUDA kernels use the same methods): accuracy against double precision,
and exact IEEE binary16 rounding against numpy."""

from __future__ import annotations

import numpy as np

from oracle import api


def _ulp_err(got: float, want: float) -> float:
    w = np.float32(want)
    u = float(np.spacing(np.abs(w)))
    return abs(got - want) / u


def test_transcendentals_accuracy():
    o = api.oracle()
    rng = np.random.Generator(np.random.PCG64(1))
    xs = np.concatenate([rng.uniform(0.003, 1.2, 4000), np.geomspace(1e-3, 4.0, 500)]).astype(np.float32)
    assert max(_ulp_err(o.oracle_cbrt(float(x)), np.cbrt(np.float64(x))) for x in xs) <= 2.0
    ps = xs[(xs > 0.04) & (xs <= 1.0)]
    assert max(_ulp_err(o.oracle_pow24(float(x)), np.float64(x) ** 2.4) for x in ps) <= 6.0
    ys = rng.uniform(-20, 20, 3000).astype(np.float32)
    assert max(_ulp_err(o.oracle_exp2(float(y)), 2.0 ** np.float64(y)) for y in ys) <= 2.0
    es = rng.uniform(-10, 10, 3000).astype(np.float32)
    assert max(_ulp_err(o.oracle_exp(float(e)), np.exp(np.float64(e))) for e in es) <= 2.0
    ls = rng.uniform(0.01, 100, 3000).astype(np.float32)
    assert max(abs(o.oracle_log2(float(v)) - np.log2(np.float64(v))) for v in ls) <= 4e-7


def test_half_conversion_exact():
    o = api.oracle()
    allh = np.arange(65536, dtype=np.uint32).astype(np.uint16)
    f = allh.view(np.float16).astype(np.float32)
    finite = np.isfinite(f)
    back = np.array([o.oracle_f2h(float(v)) for v in f[finite]], np.uint16)
    np.testing.assert_array_equal(back, allh[finite])
    rng = np.random.Generator(np.random.PCG64(2))
    vals = np.concatenate([rng.normal(0, 1e-4, 20000), rng.normal(0, 2.0, 20000), rng.uniform(-7e4, 7e4, 2000),
                           (np.arange(-3000, 3000) * 2.0 ** -25)]).astype(np.float32)
    got = np.array([o.oracle_f2h(float(v)) for v in vals], np.uint16)
    with np.errstate(over="ignore"):  # values past 65504 round to infinity, as they should
        want = vals.astype(np.float16).view(np.uint16)
    np.testing.assert_array_equal(got, want)
