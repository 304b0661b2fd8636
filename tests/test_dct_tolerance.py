"""The final DCT's contract: the stored FP16 coefficients of every first
block against the reference's formula (src/frontend_transform.cu:66-159: per
axis gf * cosf(pi (t + 1/2) k / N) with the basis rounded to float as the
reference computes it, gf = 1/N for k = 0 and sqrt(2)/N otherwise), summed
here exactly in float64 on the restatement's own sharpened planes. The
restatement sums in float with FMA in the reference's order, so it may differ
from the exact sum by the FP16 rounding (half an ulp) plus the float
accumulation error: at most 1.25 FP16 ulp is allowed. (Folding mirrored
samples, the even/odd DCT, would halve the multiply-adds but lands 9 ulp away:
the float basis is not exactly antisymmetric.) The CUDA path equals the
restatement bit for bit (tests/test_gpu_parity.py), so this pins both."""

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
    r = api.frontend(make_nv12(w, h, seed), w, h, d, debug=True)
    bw, bh = w // 8, h // 8
    nb = bw * bh
    sharp = r.sharp.reshape(3, h, w).astype(np.float64)
    coef = r.coeff.view(np.float16).astype(np.float64)
    acs = r.acs.reshape(bh, bw)
    sizes = set()
    worst = 0.0
    for by in range(bh):
        for bx in range(bw):
            n = int(acs[by, bx])
            if n == 0:
                continue
            sizes.add(n)
            D = _basis(n)
            for c in range(3):
                X = sharp[c, 8 * by:8 * by + n, 8 * bx:8 * bx + n]
                ref = (D @ X @ D.T).T  # [fx][fy]: fx across columns, fy down rows
                for raw in range(n * n):
                    fx, fy = divmod(raw, n)
                    got = coef[c * nb * 64 + P.covered_slot(n, bx, by, bw, raw)]
                    want = ref[fx, fy]
                    # Near zero the FP16 spacing is 2^-24 and the float
                    # accumulation's absolute error (a few 1e-8 times the
                    # block's sums) is allowed on top.
                    ulp = max(float(np.spacing(np.float16(abs(want)))), 2.0 ** -24)
                    worst = max(worst, (abs(got - want) - 2.0 ** -22) / ulp)
    assert sizes == {8, 16, 32}
    assert worst <= 1.25, worst
