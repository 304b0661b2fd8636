"""The final DCT's contract: the stored FP16 coefficients of every first
block against the reference's formula (src/frontend_transform.cu:66-159: per
axis gf * cosf(pi (t + 1/2) k / N) with the basis rounded to float as the
reference computes it, gf = 1/N for k = 0 and sqrt(2)/N otherwise), summed
here exactly in float64 on the restatement's own sharpened planes.

Contract: at most 1 FP16 ulp from the exact value. The only exceptions are
coefficients that the float32 sums bring near zero by cancellation: there the
FP16 spacing (down to 2^-24 in the subnormal range) is finer than the float32
accumulation's absolute error, which is bounded by 2N * 2^-24 * sum|terms|
(two passes of N products each). The reference's own kernel sums in float32
too and has the same exceptions. They are counted: under 1 in 10^4
coefficients, all below 2^-12 in magnitude, and each within 1 ulp plus that
bound. (Folding mirrored samples, the even/odd DCT, would halve the
multiply-adds but lands 9 ulp away: the float basis is not exactly
antisymmetric.) The CUDA path equals the restatement bit for bit
(tests/test_gpu_parity.py), so this pins both."""

from __future__ import annotations

import numpy as np
import pytest

from cujpegxl_b200.synth import make_nv12
from oracle import api

from . import patterns as P


def _basis(n: int) -> np.ndarray:
    """The reference's float basis gf * cosf(pi_f * (t + 0.5f) * k / n), every
    operation rounded to float (src/frontend_transform.cu:104-106)."""
    f = np.float32
    out = np.empty((n, n), np.float64)
    for k in range(n):
        gf = f(1.0) / f(n) if k == 0 else f(1.4142135623730951) / f(n)
        for t in range(n):
            arg = f(f(f(np.pi) * f(t + 0.5)) * f(k)) / f(n)
            out[k, t] = float(f(gf * f(np.cos(np.float64(arg)))))
    return out


@pytest.mark.parametrize("w,h,d,seed", [(264, 264, 1.0, 11), (520, 392, 0.5, 4)])
def test_final_dct_within_one_fp16_ulp(w, h, d, seed):
    """<= 1 FP16 ulp except near-zero cancellations (module docstring)."""
    r = api.frontend(make_nv12(w, h, seed), w, h, d, debug=True)
    bw, bh = w // 8, h // 8
    nb = bw * bh
    sharp = r.sharp.reshape(3, h, w).astype(np.float64)
    coef = r.coeff.view(np.float16).astype(np.float64)
    acs = r.acs.reshape(bh, bw)
    sizes = set()
    total = 0
    beyond = []
    for by in range(bh):
        for bx in range(bw):
            n = int(acs[by, bx])
            if n == 0:
                continue
            sizes.add(n)
            D = _basis(n)
            A = np.abs(D)
            for c in range(3):
                X = sharp[c, 8 * by:8 * by + n, 8 * bx:8 * bx + n]
                ref = (D @ X @ D.T).T  # [fx][fy]: fx across columns, fy down rows
                mag = (A @ np.abs(X) @ A.T).T
                for raw in range(n * n):
                    fx, fy = divmod(raw, n)
                    got = coef[c * nb * 64 + P.covered_slot(n, bx, by, bw, raw)]
                    want = ref[fx, fy]
                    ulp = max(float(np.spacing(np.float16(abs(want)))), 2.0 ** -24)
                    err = abs(got - want)
                    total += 1
                    if err > ulp:
                        beyond.append((err, ulp, want, mag[fx, fy], n))
    assert sizes == {8, 16, 32}
    assert len(beyond) <= total // 10000, (len(beyond), total)
    for err, ulp, want, mag, n in beyond:
        assert abs(want) < 2.0 ** -12, (err / ulp, want)
        assert err <= ulp + 2 * n * 2.0 ** -24 * mag, (err / ulp, want, mag)
