"""The frontend quantiser divides by a dequantisation weight through the
weight's rounded reciprocal (Markstein's method, `div_weight` in
cujpegxl_b200/csrc/frontend.cu). This checks, on the host's IEEE single
arithmetic, that the sequence returns the IEEE quotient for every weight of
the DCT8/16/32 tables and every significand of the dividend (which, with the
exact scaling by the dividend's exponent, is every dividend the quantiser
divides). The GPU's FMA and multiply round exactly as the host's, and the frame
parity tests compare the kernel that uses it with the restatement, which
divides."""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_weight_division_is_ieee_exhaustively(tmp_path):
    exe = tmp_path / "quant_div_check"
    subprocess.run(["gcc", "-O2", "-march=native", "-ffp-contract=off", str(REPO / "tests" / "cpu_checks" / "quant_div_check.c"),
                    "-o", str(exe), "-lm", "-lpthread"], check=True, capture_output=True, text=True, timeout=300)
    r = subprocess.run([str(exe), str(os.cpu_count() or 4)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert ", 0 mismatching quotients" in r.stdout
