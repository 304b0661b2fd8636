"""Builds libcujpegxl.so.1 (the C ABI + sm_100a kernels) in-tree.

    python -m cujpegxl_b200.build        # or build() from Python

Every .cu under csrc/ is compiled by nvcc for sm_100a only, with
-fmad=false (the kernels write every fused multiply-add explicitly, so the
float results are defined by the source alone) and host code without
contraction. The CUDA runtime is linked statically, and a version script
exports only the cujpegxl_* symbols, as the reference library does.
"""

from __future__ import annotations

import concurrent.futures
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
LIB = OUT_DIR / "libcujpegxl.so.1"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["frontend.cu", "entropy.cu", "entropy_host.cu", "cujpegxl.cu", "noalloc.cu", "batch.cu", "acsnet.cu"]
HEADERS = ["frontend.cuh", "entropy.cuh", "acsnet.cuh", "xyb.cuh", "ratio_div.cuh", "f16_mixed.cuh", "jxl_constants.cuh", "jxl_math.cuh", "prefix_code.cuh", "encoder_internal.h",
           "jxl_dequant_tables.inc", "cujpegxl.map"]


def _flags() -> list[str]:
    return ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-prec-div=true",
                   "-prec-sqrt=true", "-ftz=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
                   f"-I{REPO / 'include'}", f"-I{CSRC}"]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    OUT_DIR.mkdir(exist_ok=True)
    hdrs = [CSRC / h for h in HEADERS] + list((REPO / "include").rglob("*.h"))
    objs = []
    jobs = []
    for src in SOURCES:
        obj = OUT_DIR / (Path(src).stem + ".o")
        if force or _stale(obj, [CSRC / src] + hdrs):
            cmd = [NVCC] + _flags() + ["-c", str(CSRC / src), "-o", str(obj)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd))
            jobs.append(cmd)
        objs.append(obj)
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, len(jobs))) as pool:
        for _ in pool.map(lambda c: subprocess.run(c, check=True), jobs):
            pass
    if force or _stale(LIB, objs + [CSRC / "cujpegxl.map"]):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", str(LIB)] + [str(o) for o in objs] + [
            "-Xlinker", f"--version-script={CSRC / 'cujpegxl.map'}",
            "-Xlinker", "-soname=libcujpegxl.so.1"]
        subprocess.run(cmd, check=True)
        link = OUT_DIR / "libcujpegxl.so"
        if link.is_symlink() or link.exists():
            link.unlink()
        link.symlink_to(LIB.name)
    build_decoder(force)
    return LIB


DECODER_LIB = OUT_DIR / "libjxlsubset.so"


def build_decoder(force: bool = False) -> Path:
    """The host subset decoder (decodability and PSNR checks), g++ only."""
    OUT_DIR.mkdir(exist_ok=True)
    src = CSRC / "subset_decoder.cc"
    deps = [src, CSRC / "subset_decoder.h", CSRC / "jxl_constants.cuh", CSRC / "jxl_math.cuh",
            CSRC / "jxl_dequant_tables.inc"]
    if force or _stale(DECODER_LIB, deps):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", f"-I{CSRC}", str(src), "-o",
                        str(DECODER_LIB)], check=True)
    return DECODER_LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
