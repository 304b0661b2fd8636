"""The frontend's correctly rounded division for the adaptive-quantisation
ratios (cujpegxl_b200/csrc/ratio_div.cuh, Markstein's method on packed f32x2
arithmetic) equals IEEE division for every float argument of the ratio in
[0, 4], in both orientations. The check is compiled here for sm_100a and run
on the GPU; the frame parity tests cover the kernel that uses it."""

from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

REPO = Path(__file__).resolve().parents[1]


def test_ratio_division_is_ieee_exhaustively(tmp_path):
    from cujpegxl_b200 import build as B

    exe = tmp_path / "ratio_div_check"
    subprocess.run([B.NVCC, *B.ARCH, "-O3", "-std=c++17", "-fmad=false", "-I", str(B.CSRC),
                    str(REPO / "tests" / "gpu_checks" / "ratio_div_check.cu"), "-o", str(exe)],
                   check=True, capture_output=True, text=True, timeout=600)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "num/den mismatches 0, den/num mismatches 0" in r.stdout
