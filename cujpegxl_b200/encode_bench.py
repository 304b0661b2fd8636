"""Command-line encode benchmark with the reference tool's flags and report.

    python -m cujpegxl_b200.encode_bench --codec=<cujpegxl|nvjpeg> --dims=WxH [options] f1.nv12 [...]

The same interface as the reference's `encode_bench`
(tools/benchmark/encode_bench.cc:46-69): the flags, their defaults, the
validation messages and the stdout report (encode_bench.cc:361-390) are the
reference's, so its driver and parser (tools/benchmark/benchmark.py:76-102)
run unchanged against this module.

NV12 files (width*height*3/2 bytes each, all of the same --dims) are read once
and uploaded once; each timed iteration is one device-resident encode, the
iterations alternating across the files. `--codec=cujpegxl` times one
`cujpegxl_encoder_encode` call through the C ABI (device NV12 in, host .jxl
bytes out, the device-to-host read of the file included), with a device
synchronise before and after, on the host clock, as encode_bench.cc:462-472
and :517-525 do. `--codec=nvjpeg` times nvjpegEncodeYUV plus the bitstream
read-back on planar Y/Cb/Cr (the chroma de-interleaved once at load), as
encode_bench.cc:476-494 does; it is the vendor baseline the reference compares
against, called from the CUDA toolkit's libnvjpeg.

`--profile` (cujpegxl only) defaults the iteration count to 1 and, after the
timed loop, runs the last iteration's frame once more stage by stage and
prints one record per stage in the reference's layout (encode_bench.cc:
528-546): `frontend` (the fused frontend kernel), `entropy` (histograms,
codes, token emission and the device-side headers/TOC/container) and
`assembly` (reading the finished file back to the host). `bytes` is each
stage's algorithmic DRAM traffic. Every encode is wrapped in an NVTX range
named `cujpegxl_encode` / `nvjpeg_encode`.
"""

from __future__ import annotations

import ctypes
import math
import re
import sys
import time
from dataclasses import dataclass, field

import numpy as np

USAGE = (
    "encode_bench: measure GPU encode time of NV12 images with cujpegxl or nvJPEG.\n"
    "\n"
    "Usage:\n"
    "  python -m cujpegxl_b200.encode_bench --codec=<cujpegxl|nvjpeg> --dims=WxH [options] <file1.nv12> [...]\n"
    "\n"
    "Options:\n"
    "  --codec=<cujpegxl|nvjpeg>   Encoder to benchmark (required).\n"
    "  --dims=WxH                  Frame dimensions in pixels (required).\n"
    "  --iterations=N              Timed encode iterations (default 5).\n"
    "  --warmup=N                  Untimed warmup encode iterations (default 1).\n"
    "  --distance=F                cujpegxl Butteraugli distance (default 1.0).\n"
    "  --quality=N                 nvJPEG quality 1..100 (default 90).\n"
    "  --device=N                  CUDA device ordinal (default 0).\n"
    "  --profile                   cujpegxl only: defaults iterations to 1 (unless\n"
    "                              --iterations is given explicitly), wraps each\n"
    "                              encode in an NVTX range, and prints per-stage\n"
    "                              timings for the final iteration.\n"
    "  -h, --help                  Show this help.\n"
)


class BenchError(SystemExit):
    """Raised by die(): the message goes to stderr and the exit status is 1."""


def die(msg: str):
    print(f"encode_bench: {msg}", file=sys.stderr)
    raise BenchError(1)


@dataclass
class Args:
    codec: str = ""
    width: int = 0
    height: int = 0
    iterations: int = 5
    warmup: int = 1
    distance: float = 1.0
    quality: int = 90
    device: int = 0
    profile: bool = False
    iterations_explicit: bool = False
    files: list[str] = field(default_factory=list)


def _parse_int(s: str) -> int | None:
    """strtol base 10 with the whole string consumed: leading white space,
    an optional sign, digits."""
    m = re.fullmatch(r"\s*([+-]?\d+)", s)
    return int(m.group(1)) if m else None


def _parse_float(s: str) -> float | None:
    if "_" in s:
        return None
    try:
        v = float(s)
    except ValueError:
        return None
    # strtof overflows to ERANGE for values beyond float's range.
    if math.isfinite(v) and abs(v) > 3.4028234663852886e38:
        return None
    return float(np.float32(v))


def parse_args(argv: list[str]) -> Args:
    """Flag parsing as encode_bench.cc:128-206: `--flag=value` or `--flag value`,
    anything else that starts with `--` is an error, the rest are files."""
    a = Args()
    i = 0

    def take_value(arg: str) -> str:
        nonlocal i
        eq = arg.find("=")
        if eq >= 0:
            return arg[eq + 1:]
        if i + 1 < len(argv):
            i += 1
            return argv[i]
        die("missing value for " + arg)

    while i < len(argv):
        arg = argv[i]
        if arg in ("-h", "--help"):
            print(USAGE)
            raise SystemExit(0)
        elif arg.startswith("--codec"):
            a.codec = take_value(arg)
        elif arg.startswith("--dims"):
            v = take_value(arg)
            x = v.find("x")
            if x < 0:
                die("expected --dims=WxH, got: " + v)
            w, h = _parse_int(v[:x]), _parse_int(v[x + 1:])
            if w is None or h is None or w <= 0 or h <= 0:
                die("invalid dims: " + v)
            a.width, a.height = w, h
        elif arg.startswith("--iterations"):
            v = _parse_int(take_value(arg))
            if v is None:
                die("--iterations requires an integer")
            a.iterations, a.iterations_explicit = v, True
        elif arg.startswith("--warmup"):
            v = _parse_int(take_value(arg))
            if v is None:
                die("--warmup requires an integer")
            a.warmup = v
        elif arg.startswith("--distance"):
            f = _parse_float(take_value(arg))
            if f is None:
                die("--distance requires a number")
            a.distance = f
        elif arg.startswith("--quality"):
            v = _parse_int(take_value(arg))
            if v is None:
                die("--quality requires an integer")
            a.quality = v
        elif arg.startswith("--device"):
            v = _parse_int(take_value(arg))
            if v is None:
                die("--device requires an integer")
            a.device = v
        elif arg == "--profile":
            a.profile = True
        elif arg.startswith("--"):
            die("unknown option: " + arg)
        else:
            a.files.append(arg)
        i += 1
    return a


def validate(a: Args) -> Args:
    """The checks of encode_bench.cc:396-431, in the same order and words."""
    if not a.codec:
        die("--codec=<cujpegxl|nvjpeg> is required")
    if a.codec not in ("cujpegxl", "nvjpeg"):
        die("--codec must be 'cujpegxl' or 'nvjpeg'")
    if a.width == 0 or a.height == 0:
        die("--dims=WxH is required")
    if not a.files:
        die("at least one NV12 input file is required")
    if a.width % 2 or a.height % 2:
        die("dims must be even (NV12 4:2:0 constraint)")
    if a.width % 8 or a.height % 8:
        die("dims must be multiples of 8 (cujpegxl block size constraint)")
    if a.iterations < 1:
        die("--iterations must be >= 1")
    if a.warmup < 0:
        die("--warmup must be >= 0")
    if a.profile and a.codec != "cujpegxl":
        die("--profile is only supported with --codec=cujpegxl")
    if a.profile and not a.iterations_explicit:
        a.iterations = 1
    if a.codec == "cujpegxl" and not (a.distance > 0.0 and math.isfinite(a.distance)):
        die("--distance must be a positive finite number")
    if a.codec == "nvjpeg" and not (1 <= a.quality <= 100):
        die("--quality must be in [1, 100]")
    return a


def load_nv12(path: str, width: int, height: int) -> np.ndarray:
    expected = width * height * 3 // 2
    try:
        with open(path, "rb") as f:
            data = f.read(expected)
    except OSError:
        die("cannot open: " + path)
    if len(data) != expected:
        die(f"short read on {path}: expected {expected} bytes")
    return np.frombuffer(data, np.uint8)


def deinterleave_chroma(nv12: np.ndarray, width: int, height: int) -> tuple[np.ndarray, np.ndarray]:
    """NV12's interleaved Cb/Cr plane as two planar (height/2, width/2) planes."""
    uv = nv12[width * height:].reshape(height // 2, width // 2, 2)
    return np.ascontiguousarray(uv[..., 0]), np.ascontiguousarray(uv[..., 1])


def mean_of(xs: list[float]) -> float:
    return sum(xs) / len(xs)


def stddev_of(xs: list[float]) -> float:
    if len(xs) < 2:
        return 0.0
    m = mean_of(xs)
    return math.sqrt(sum((x - m) ** 2 for x in xs) / (len(xs) - 1))


def percentile_of(xs: list[float], p: float) -> float:
    """Nearest-rank on the sorted samples, index llround(p * (n - 1))."""
    s = sorted(xs)
    return s[int(math.floor(p * (len(s) - 1) + 0.5))]


def header_lines(a: Args, image_count: int) -> list[str]:
    lines = [
        "encode_bench",
        f"  codec:      {a.codec}",
        f"  dims:       {a.width}x{a.height}",
        f"  images:     {image_count}",
        f"  iterations: {a.iterations}",
        f"  warmup:     {a.warmup}",
    ]
    if a.codec == "cujpegxl":
        lines.append(f"  distance:   {a.distance:.2f}")
    else:
        lines.append(f"  quality:    {a.quality}")
    lines.append(f"  device:     {a.device}")
    lines.append(f"  profile:    {'true' if a.profile else 'false'}")
    return lines


def stats_lines(times_us: list[float], codec: str) -> list[str]:
    total = sum(times_us)
    mean = mean_of(times_us)
    fps = 1.0e6 / mean if mean > 0.0 else 0.0
    return [
        "",
        f"results ({codec}, microseconds):",
        f"  n:          {len(times_us)}",
        f"  total:      {total:.0f}",
        f"  mean:       {mean:.0f}   ({fps:.2f} fps)",
        f"  stddev:     {stddev_of(times_us):.0f}",
        f"  min:        {min(times_us):.0f}",
        f"  p50:        {percentile_of(times_us, 0.50):.0f}",
        f"  p99:        {percentile_of(times_us, 0.99):.0f}",
        f"  max:        {max(times_us):.0f}",
    ]


def stage_lines(stages: list[dict], a: Args) -> list[str]:
    lines = ["", "cujpegxl per-stage timings (last iteration):"]
    for s in stages:
        lines.append(f"  {s['name']:<10} gpu={s['gpu_us']:9.0f} us  cpu={s['cpu_us']:7.0f} us  bytes={s['bytes_moved']}")
    first = a.files[0]
    lines += [
        "",
        "Capture a detailed profile with:",
        f"  ncu --clock-control none --set full -k regex:frontend_kernel -c 1 python -m cujpegxl_b200.encode_bench "
        f"--codec=cujpegxl --dims={a.width}x{a.height} --profile {first}",
    ]
    return lines


def stage_bytes(width: int, height: int, file_size: int) -> dict[str, int]:
    """Algorithmic DRAM bytes per stage: the frontend reads NV12 and writes
    int16 AC, int32 DC, the transform map, the int32 quant field and the CfL
    maps; entropy reads those planes and writes the file; assembly moves the
    file to the host."""
    p = width * height
    b = p // 64
    t = ((width // 8 + 7) // 8) * ((height // 8 + 7) // 8)
    planes = 6 * p + 12 * b + 5 * b + 2 * t
    return {"frontend": int(1.5 * p) + planes, "entropy": planes + file_size, "assembly": file_size}


class Nvjpeg:
    """The vendor JPEG encoder through the CUDA toolkit's libnvjpeg: one
    handle, encoder state and parameter set reused across iterations, 4:2:0
    planar input, the default stream (encode_bench.cc:319-355)."""

    CSS_420 = 2
    MAX_COMPONENT = 4

    class Image(ctypes.Structure):
        _fields_ = [("channel", ctypes.c_void_p * 4), ("pitch", ctypes.c_size_t * 4)]

    def __init__(self, quality: int, width: int, height: int):
        self.L = ctypes.CDLL("libnvjpeg.so.12")
        vp = ctypes.c_void_p
        self.handle, self.state, self.params = vp(), vp(), vp()
        self._check(self.L.nvjpegCreateSimple(ctypes.byref(self.handle)), "CreateSimple")
        self._check(self.L.nvjpegEncoderStateCreate(self.handle, ctypes.byref(self.state), vp()), "EncoderStateCreate")
        self._check(self.L.nvjpegEncoderParamsCreate(self.handle, ctypes.byref(self.params), vp()),
                    "EncoderParamsCreate")
        self._check(self.L.nvjpegEncoderParamsSetQuality(self.params, ctypes.c_int(quality), vp()), "SetQuality")
        self._check(self.L.nvjpegEncoderParamsSetSamplingFactors(self.params, ctypes.c_int(self.CSS_420), vp()),
                    "SetSamplingFactors")
        size = ctypes.c_size_t(0)
        self._check(self.L.nvjpegEncodeGetBufferSize(self.handle, self.params, ctypes.c_int(width),
                                                     ctypes.c_int(height), ctypes.byref(size)),
                    "EncodeGetBufferSize")
        self.output = np.zeros(size.value, np.uint8)
        self.image = self.Image()

    @staticmethod
    def _check(status: int, what: str) -> None:
        if status != 0:
            die(f"nvjpeg {what} failed (status {status})")

    def encode(self, y: int, cb: int, cr: int, width: int, height: int) -> int:
        img = self.image
        img.channel[0], img.pitch[0] = y, width
        img.channel[1], img.pitch[1] = cb, width // 2
        img.channel[2], img.pitch[2] = cr, width // 2
        vp = ctypes.c_void_p
        self._check(self.L.nvjpegEncodeYUV(self.handle, self.state, self.params, ctypes.byref(img),
                                           ctypes.c_int(self.CSS_420), ctypes.c_int(width), ctypes.c_int(height),
                                           vp()), "EncodeYUV")
        length = ctypes.c_size_t(self.output.size)
        self._check(self.L.nvjpegEncodeRetrieveBitstream(self.handle, self.state,
                                                         ctypes.c_void_p(self.output.ctypes.data),
                                                         ctypes.byref(length), vp()), "RetrieveBitstream")
        return length.value

    def close(self) -> None:
        if self.params:
            self.L.nvjpegEncoderParamsDestroy(self.params)
            self.params = ctypes.c_void_p()
        if self.state:
            self.L.nvjpegEncoderStateDestroy(self.state)
            self.state = ctypes.c_void_p()
        if self.handle:
            self.L.nvjpegDestroy(self.handle)
            self.handle = ctypes.c_void_p()


def _copy_to_host(dst: np.ndarray, src_device: int, size: int) -> None:
    from cuda.bindings import runtime as rt

    (err,) = rt.cudaMemcpy(dst.ctypes.data, src_device, size, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    if err != rt.cudaError_t.cudaSuccess:
        die(f"cuda memcpy failed: {err}")


def profile_stages(enc, luma: int, chroma: int, width: int, height: int) -> list[dict]:
    """One more encode of the frame, stage by stage, each stage synchronised
    and timed on the host clock like the timed loop."""
    import torch

    from . import _capi

    out = []
    # The first runtime call of the copy path loads its bindings; keep that
    # out of the assembly record.
    size, dev = enc.result()
    _copy_to_host(np.empty(max(size, 1), np.uint8), dev, min(size, 1))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    enc.enqueue_stages(luma, chroma, width, width, _capi.STAGE_FRONTEND)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    enc.enqueue_stages(luma, chroma, width, width, _capi.STAGE_ENTROPY)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    size, dev = enc.result()
    host = np.empty(size, np.uint8)
    _copy_to_host(host, dev, size)
    t3 = time.perf_counter()
    nbytes = stage_bytes(width, height, size)
    out.append({"name": "frontend", "bytes_moved": nbytes["frontend"], "gpu_us": (t1 - t0) * 1e6, "cpu_us": 0.0})
    out.append({"name": "entropy", "bytes_moved": nbytes["entropy"], "gpu_us": (t2 - t1) * 1e6, "cpu_us": 0.0})
    out.append({"name": "assembly", "bytes_moved": nbytes["assembly"], "gpu_us": 0.0, "cpu_us": (t3 - t2) * 1e6})
    return out


def run(a: Args) -> int:
    import torch

    from . import Encoder

    if not torch.cuda.is_available():
        die("cuda cudaSetDevice failed: no CUDA device")
    if a.device < 0 or a.device >= torch.cuda.device_count():
        die(f"cuda cudaSetDevice failed: invalid device ordinal {a.device}")
    dev = torch.device("cuda", a.device)
    torch.cuda.set_device(dev)
    torch.cuda.synchronize()

    W, H = a.width, a.height
    images = []
    for path in a.files:
        nv12 = load_nv12(path, W, H)
        if a.codec == "cujpegxl":
            luma = torch.from_numpy(nv12[: W * H].copy()).to(dev)
            chroma = torch.from_numpy(nv12[W * H:].copy()).to(dev)
            images.append((luma, chroma))
        else:
            cb, cr = deinterleave_chroma(nv12, W, H)
            y = torch.from_numpy(nv12[: W * H].copy()).to(dev)
            images.append((y, torch.from_numpy(cb).to(dev), torch.from_numpy(cr).to(dev)))
    torch.cuda.synchronize()

    print("\n".join(header_lines(a, len(images))), flush=True)

    enc = nvj = None
    if a.codec == "cujpegxl":
        enc = Encoder(W, H, a.distance, a.device)
    else:
        nvj = Nvjpeg(a.quality, W, H)

    def encode_one(img) -> float:
        torch.cuda.nvtx.range_push("cujpegxl_encode" if enc is not None else "nvjpeg_encode")
        t0 = time.perf_counter()
        if enc is not None:
            enc.encode_device(img[0].data_ptr(), img[1].data_ptr(), W, W)
        else:
            nvj.encode(img[0].data_ptr(), img[1].data_ptr(), img[2].data_ptr(), W, H)
            torch.cuda.synchronize()
        us = (time.perf_counter() - t0) * 1e6
        torch.cuda.nvtx.range_pop()
        return us

    try:
        for w in range(a.warmup):
            encode_one(images[w % len(images)])
        torch.cuda.synchronize()

        times_us = []
        for i in range(a.iterations):
            img = images[i % len(images)]
            torch.cuda.synchronize()
            us = encode_one(img)
            torch.cuda.synchronize()
            times_us.append(us)
            print(f"[{a.codec}] iter {i + 1}/{a.iterations}: {us:.0f} us", file=sys.stderr)

        print("\n".join(stats_lines(times_us, a.codec)), flush=True)

        if a.profile and enc is not None:
            img = images[(a.iterations - 1) % len(images)]
            stages = profile_stages(enc, img[0].data_ptr(), img[1].data_ptr(), W, H)
            print("\n".join(stage_lines(stages, a)), flush=True)
    finally:
        if enc is not None:
            enc.close()
        if nvj is not None:
            nvj.close()
    return 0


def main(argv: list[str] | None = None) -> int:
    a = validate(parse_args(sys.argv[1:] if argv is None else argv))
    return run(a)


if __name__ == "__main__":
    raise SystemExit(main())
