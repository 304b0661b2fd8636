"""The encode_bench command line on the GPU: both codecs run over several
NV12 files, alternate across them and print a report that the reference's
parser reads back; --profile prints the three stage records; the nvJPEG
baseline writes a JPEG stream."""

from __future__ import annotations

import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from cujpegxl_b200 import encode_bench as eb
from cujpegxl_b200.synth import make_nv12

from .test_encode_bench_cli import _parse_like_reference

pytestmark = pytest.mark.gpu

REPO = Path(__file__).resolve().parents[1]
W, H = 512, 384


def _files(tmp_path, count):
    paths = []
    for i in range(count):
        p = tmp_path / f"frame{i}.nv12"
        p.write_bytes(make_nv12(W, H, i).tobytes())
        paths.append(str(p))
    return paths


def _run(args):
    r = subprocess.run([sys.executable, "-m", "cujpegxl_b200.encode_bench", *args], cwd=REPO,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r


@pytest.mark.parametrize("codec", ["cujpegxl", "nvjpeg"])
def test_cli_reports(tmp_path, codec):
    files = _files(tmp_path, 2)
    r = _run(["--codec", codec, "--dims", f"{W}x{H}", "--iterations", "5", "--warmup", "2", *files])
    s = _parse_like_reference(r.stdout)
    assert (s["codec"], s["width"], s["height"], s["images"], s["n"]) == (codec, W, H, 2, 5)
    assert 0 < s["min"] <= s["p50"] <= s["max"] and s["fps"] > 0
    iters = re.findall(rf"\[{codec}\] iter (\d+)/5: \d+ us", r.stderr)
    assert iters == ["1", "2", "3", "4", "5"]


def test_cli_profile_stages(tmp_path):
    files = _files(tmp_path, 1)
    r = _run(["--codec=cujpegxl", f"--dims={W}x{H}", "--profile", *files])
    assert _parse_like_reference(r.stdout)["n"] == 1
    stages = re.findall(r"^  (\w+)\s+gpu=\s*(\d+) us  cpu=\s*(\d+) us  bytes=(\d+)$", r.stdout, re.M)
    assert [s[0] for s in stages] == ["frontend", "entropy", "assembly"]
    assert int(stages[0][3]) == eb.stage_bytes(W, H, 0)["frontend"]


def test_nvjpeg_baseline_writes_jpeg():
    import torch

    nv12 = make_nv12(W, H, 5)
    cb, cr = eb.deinterleave_chroma(nv12, W, H)
    assert np.array_equal(cb[1, 3], nv12[W * H + W + 6]) and np.array_equal(cr[1, 3], nv12[W * H + W + 7])
    y = torch.from_numpy(nv12[: W * H].copy()).cuda()
    tcb, tcr = torch.from_numpy(cb).cuda(), torch.from_numpy(cr).cuda()
    torch.cuda.synchronize()
    nvj = eb.Nvjpeg(90, W, H)
    try:
        n = nvj.encode(y.data_ptr(), tcb.data_ptr(), tcr.data_ptr(), W, H)
        torch.cuda.synchronize()
        data = nvj.output[:n].tobytes()
    finally:
        nvj.close()
    assert data[:2] == b"\xff\xd8" and data[-2:] == b"\xff\xd9"
