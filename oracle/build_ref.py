"""Build recipe for oracle/_ref/libjxlref.so: the reference's own host code.

Test infrastructure only. Compiles, where they lie under the reference
checkout, the reference's host-compilable sources (its bitstream writer, host
bitstream reference, coefficient order and VarDCT layout) together with
oracle/ref_shim.cc, which exposes C entry points over them and over the
reference's host/device helper headers. Nothing is copied out of the
reference tree; the only output is the shared library in oracle/_ref/.

The reference's CUDA translation units are not built: three of them do not
compile with nvcc unmodified, and its build system (Bazel with an
un-vendored libjxl) is not used.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
# The reference checkout: CUJPEGXL_REFERENCE, else a "reference" directory
# beside this repository's root.
REFERENCE = Path(os.environ.get("CUJPEGXL_REFERENCE", HERE.parent.parent / "reference"))
OUT_DIR = HERE / "_ref"
OUT = OUT_DIR / "libjxlref.so"

SOURCES = [
    "src/bitstream/prefix_code.cc",
    "src/bitstream/context_map.cc",
    "src/bitstream/histogram_writer.cc",
    "src/bitstream/frame_assembly.cc",
    "src/bitstream/codestream.cc",
    "src/bitstream/container.cc",
    "tools/bitstream/vardct_frame.cc",
    "tools/bitstream/entropy_encoder.cc",
    "tools/bitstream/modular.cc",
    "src/coeff_order.cc",
    "src/vardct_layout.cc",
]

CUDA_INCLUDE = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "include"


def available() -> bool:
    return (REFERENCE / "src" / "bitstream" / "prefix_code.cc").is_file()


def build(force: bool = False) -> Path | None:
    """Builds the library if the reference checkout is present; returns its path."""
    if not available():
        return OUT if OUT.exists() else None
    srcs = [REFERENCE / s for s in SOURCES] + [HERE / "ref_shim.cc"]
    if OUT.exists() and not force:
        newest = max(p.stat().st_mtime for p in srcs)
        if OUT.stat().st_mtime >= newest:
            return OUT
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    cmd = [
        "g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-ffp-contract=off",
        f"-I{REFERENCE}", f"-I{CUDA_INCLUDE}", "-o", str(OUT),
    ] + [str(s) for s in srcs]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    path = build(force="--force" in sys.argv)
    print(path if path else "reference not present; nothing built")
