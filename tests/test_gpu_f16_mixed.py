"""The mixed-precision FP16-input instructions that carry the frontend's
chroma-from-luma sums (cujpegxl_b200/csrc/f16_mixed.cuh: fma.rn.f32.f16 and
add.rn.f32.f16) give exactly the convert-then-FP32 results the CPU
restatement computes, for every ordered pair of finite FP16 operands. The
check is compiled here for sm_100a and run on the GPU."""

from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

REPO = Path(__file__).resolve().parents[1]


def test_mixed_precision_equals_convert_then_fp32(tmp_path):
    from cujpegxl_b200 import build as B

    exe = tmp_path / "f16_mixed_check"
    subprocess.run([B.NVCC, *B.ARCH, "-O3", "-std=c++17", "-fmad=false", "-I", str(B.CSRC),
                    str(REPO / "tests" / "gpu_checks" / "f16_mixed_check.cu"), "-o", str(exe)],
                   check=True, capture_output=True, text=True, timeout=600)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fma mismatches 0, sub mismatches 0, add mismatches 0" in r.stdout
