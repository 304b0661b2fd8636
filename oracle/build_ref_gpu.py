"""Build recipe for oracle/_ref/libjxlref_gpu.so: the reference's own device
code for the float stages, as a checker on a GPU.

Test infrastructure only. nvcc compiles, where they lie under the reference
checkout, the reference's CUDA translation units that it accepts unchanged
(src/xyb.cu, src/frontend_fused.cu, src/frontend_transform.cu) for sm_100a
with nvcc's default floating-point contraction, and oracle/ref_gpu_shim.cc,
which exposes C entry points over them. Nothing is copied out of the
reference tree; the only output is the shared library in oracle/_ref/.

src/transform_select.cu, src/frontend_quantize.cu and src/entropy.cu are not
built: they read constexpr host tables from device code, which the
reference's own CUDA compiler (clang) accepts and nvcc does not.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from build_ref import REFERENCE  # noqa: E402  (sibling module: the reference's location)

OUT_DIR = HERE / "_ref"
OUT = OUT_DIR / "libjxlref_gpu.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_INCLUDE = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "include"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["src/xyb.cu", "src/frontend_fused.cu", "src/frontend_transform.cu"]


def available() -> bool:
    return all((REFERENCE / s).is_file() for s in SOURCES)


def build(force: bool = False) -> Path | None:
    """Builds the library if the reference checkout is present; returns its path."""
    if not available():
        return OUT if OUT.exists() else None
    srcs = [REFERENCE / s for s in SOURCES] + [HERE / "ref_gpu_shim.cc"]
    if OUT.exists() and not force:
        if OUT.stat().st_mtime >= max(p.stat().st_mtime for p in srcs + [Path(__file__)]):
            return OUT
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    objs = []
    for s in srcs[:-1]:
        obj = OUT_DIR / (s.stem + "_gpu.o")
        subprocess.run([NVCC] + ARCH + ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", f"-I{REFERENCE / 'src'}",
                                        "-c", str(s), "-o", str(obj)], check=True)
        objs.append(obj)
    # The shim is host code (it includes the reference's host decision code).
    shim = OUT_DIR / "ref_gpu_shim.o"
    subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", f"-I{REFERENCE}",
                    f"-I{CUDA_INCLUDE}", "-c", str(srcs[-1]), "-o", str(shim)], check=True)
    objs.append(shim)
    subprocess.run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", str(OUT)] + [str(o) for o in objs],
                   check=True)
    for o in objs:
        o.unlink()
    return OUT


if __name__ == "__main__":
    path = build(force="--force" in sys.argv)
    print(path if path else "reference not present; nothing built")
