"""Builds the CPU restatement (oracle/liboracle.so) and, when the reference
checkout is present, the reference checker libraries (oracle/_ref/libjxlref.so
from its host code, oracle/_ref/libjxlref_gpu.so from its device code).

Test infrastructure only. The restatement is compiled without floating-point
contraction so that fmaf appears exactly where the source writes it.
"""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
SOURCES = [HERE / "frontend_oracle.c", HERE / "bitstream_oracle.c"]
DEPS = SOURCES + [HERE / "oracle.h", HERE.parent / "cujpegxl_b200" / "csrc" / "jxl_dequant_tables.inc"]


def build_oracle(force: bool = False) -> Path:
    if LIB.exists() and not force:
        if LIB.stat().st_mtime >= max(p.stat().st_mtime for p in DEPS):
            return LIB
    cmd = ["gcc", "-std=gnu11", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
           "-pthread", "-o", str(LIB)] + [str(s) for s in SOURCES] + ["-lm"]
    subprocess.run(cmd, check=True)
    return LIB


def build(force: bool = False) -> None:
    build_oracle(force)
    sys.path.insert(0, str(HERE))
    import build_ref  # noqa: E402  (sibling module)
    import build_ref_gpu  # noqa: E402

    build_ref.build(force)
    build_ref_gpu.build(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(LIB)
