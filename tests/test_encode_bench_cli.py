"""The encode_bench command line without a GPU: flag parsing and validation
with the reference tool's messages and exit codes
(tools/benchmark/encode_bench.cc:128-206, :396-431), and a report that the
reference's own parser reads back (tools/benchmark/benchmark.py:76-102,
whose patterns are restated here)."""

from __future__ import annotations

import re

import numpy as np
import pytest

from cujpegxl_b200 import encode_bench as eb


def _die_message(capsys, argv) -> str:
    with pytest.raises(SystemExit) as exc:
        eb.validate(eb.parse_args(argv))
    assert exc.value.code == 1
    return capsys.readouterr().err.strip()


@pytest.mark.parametrize("argv,msg", [
    ([], "--codec=<cujpegxl|nvjpeg> is required"),
    (["--codec=webp", "--dims=64x64", "a"], "--codec must be 'cujpegxl' or 'nvjpeg'"),
    (["--codec=cujpegxl", "a"], "--dims=WxH is required"),
    (["--codec=cujpegxl", "--dims=64x64"], "at least one NV12 input file is required"),
    (["--codec=cujpegxl", "--dims=66x63", "a"], "dims must be even (NV12 4:2:0 constraint)"),
    (["--codec=cujpegxl", "--dims=68x64", "a"], "dims must be multiples of 8 (cujpegxl block size constraint)"),
    (["--codec=cujpegxl", "--dims=64x64", "--iterations=0", "a"], "--iterations must be >= 1"),
    (["--codec=cujpegxl", "--dims=64x64", "--warmup=-1", "a"], "--warmup must be >= 0"),
    (["--codec=nvjpeg", "--dims=64x64", "--profile", "a"], "--profile is only supported with --codec=cujpegxl"),
    (["--codec=cujpegxl", "--dims=64x64", "--distance=0", "a"], "--distance must be a positive finite number"),
    (["--codec=cujpegxl", "--dims=64x64", "--distance=inf", "a"], "--distance must be a positive finite number"),
    (["--codec=nvjpeg", "--dims=64x64", "--quality=101", "a"], "--quality must be in [1, 100]"),
    (["--codec=cujpegxl", "--dims=64"], "expected --dims=WxH, got: 64"),
    (["--codec=cujpegxl", "--dims=0x64"], "invalid dims: 0x64"),
    (["--codec=cujpegxl", "--dims=6ax64"], "invalid dims: 6ax64"),
    (["--iterations=x"], "--iterations requires an integer"),
    (["--warmup", "1.5"], "--warmup requires an integer"),
    (["--distance=abc"], "--distance requires a number"),
    (["--distance=1e39"], "--distance requires a number"),
    (["--quality="], "--quality requires an integer"),
    (["--device=zero"], "--device requires an integer"),
    (["--frobnicate"], "unknown option: --frobnicate"),
    (["--codec"], "missing value for --codec"),
])
def test_validation_messages(capsys, argv, msg):
    assert _die_message(capsys, argv) == f"encode_bench: {msg}"


def test_flag_forms_and_defaults():
    a = eb.validate(eb.parse_args(["--codec", "cujpegxl", "--dims", "3840x2160", "f1", "f2"]))
    assert (a.codec, a.width, a.height, a.iterations, a.warmup, a.distance, a.quality, a.device, a.profile) == \
        ("cujpegxl", 3840, 2160, 5, 1, 1.0, 90, 0, False)
    assert a.files == ["f1", "f2"]
    # The driver's own command form (benchmark.py:146-160).
    a = eb.validate(eb.parse_args(["--codec", "nvjpeg", "--dims", "1920x1080", "--iterations", "10", "--warmup",
                                   "2", "--device", "0", "--quality", "75", "x.nv12"]))
    assert (a.iterations, a.warmup, a.quality) == (10, 2, 75)
    # --profile drops the default iteration count to 1, not an explicit one.
    assert eb.validate(eb.parse_args(["--codec=cujpegxl", "--dims=64x64", "--profile", "f"])).iterations == 1
    assert eb.validate(eb.parse_args(["--codec=cujpegxl", "--dims=64x64", "--iterations=4", "--profile",
                                      "f"])).iterations == 4
    # strtof rounds to float.
    assert eb.parse_args(["--distance=0.1"]).distance == float(np.float32(0.1))


def test_help_exits_zero(capsys):
    with pytest.raises(SystemExit) as exc:
        eb.parse_args(["--help"])
    assert exc.value.code == 0
    assert "--codec=<cujpegxl|nvjpeg>" in capsys.readouterr().out


def test_statistics_match_the_reference_definitions():
    rng = np.random.default_rng(3)
    for n in (1, 2, 5, 100, 101):
        xs = list(rng.uniform(100, 5000, n))
        assert eb.mean_of(xs) == pytest.approx(np.mean(xs))
        assert eb.stddev_of(xs) == pytest.approx(np.std(xs, ddof=1) if n > 1 else 0.0)
        s = sorted(xs)
        for p in (0.5, 0.99):
            # std::llround(p * (n - 1)) rounds halves away from zero.
            idx = int(np.floor(p * (n - 1) + 0.5))
            assert eb.percentile_of(xs, p) == s[idx]


def _parse_like_reference(out: str) -> dict:
    def field(pattern: str) -> re.Match:
        m = re.search(pattern, out)
        assert m is not None, pattern
        return m

    mean = field(r"mean:\s+([\d.]+)\s+\(([\d.]+) fps\)")
    r = {
        "codec": field(r"codec:\s+(\S+)").group(1),
        "width": int(field(r"dims:\s+(\d+)x\d+").group(1)),
        "height": int(field(r"dims:\s+\d+x(\d+)").group(1)),
        "images": int(field(r"images:\s+(\d+)").group(1)),
        "iterations": int(field(r"iterations:\s+(\d+)").group(1)),
        "warmup": int(field(r"warmup:\s+(\d+)").group(1)),
        "n": int(field(r"\bn:\s+(\d+)").group(1)),
        "total": float(field(r"total:\s+([\d.]+)").group(1)),
        "mean": float(mean.group(1)),
        "fps": float(mean.group(2)),
        "stddev": float(field(r"stddev:\s+([\d.]+)").group(1)),
        "min": float(field(r"min:\s+([\d.]+)").group(1)),
        "p50": float(field(r"p50:\s+([\d.]+)").group(1)),
        "p99": float(field(r"p99:\s+([\d.]+)").group(1)),
        "max": float(field(r"max:\s+([\d.]+)").group(1)),
    }
    if r["codec"] == "cujpegxl":
        r["setting"] = f"d={float(field(r'distance:\s+([\d.]+)').group(1))}"
    else:
        r["setting"] = f"q={int(field(r'quality:\s+(\d+)').group(1))}"
    return r


@pytest.mark.parametrize("codec", ["cujpegxl", "nvjpeg"])
def test_report_reads_back_with_the_reference_parser(codec):
    a = eb.validate(eb.parse_args([f"--codec={codec}", "--dims=3840x2160", "--iterations=4", "f1", "f2"]))
    times = [1100.4, 1050.0, 990.6, 1201.2]
    out = "\n".join(eb.header_lines(a, 2) + eb.stats_lines(times, codec))
    r = _parse_like_reference(out)
    assert (r["codec"], r["width"], r["height"], r["images"], r["iterations"], r["warmup"], r["n"]) == \
        (codec, 3840, 2160, 2, 4, 1, 4)
    assert r["setting"] == ("d=1.0" if codec == "cujpegxl" else "q=90")
    assert r["total"] == round(sum(times))
    assert r["mean"] == round(np.mean(times))
    assert r["fps"] == pytest.approx(1e6 / np.mean(times), abs=0.005)
    assert (r["min"], r["max"]) == (round(min(times)), round(max(times)))


def test_stage_bytes():
    b = eb.stage_bytes(3840, 2160, 1000)
    p = 3840 * 2160
    assert b["frontend"] > 7 * p and b["entropy"] > 6 * p and b["assembly"] == 1000


def test_run_without_a_device_fails_loudly(capsys, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    f = tmp_path / "f.nv12"
    f.write_bytes(bytes(64 * 64 * 3 // 2))
    with pytest.raises(SystemExit) as exc:
        eb.main(["--codec=cujpegxl", "--dims=64x64", str(f)])
    assert exc.value.code == 1
    assert capsys.readouterr().err.startswith("encode_bench: cuda")
