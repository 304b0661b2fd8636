"""Deterministic quantised-plane patterns for entropy-stage tests.

Restated from the reference's entropy tests so the same coverage applies:
the AC pattern of src/entropy_gpu_test.cc:53-73 (small and large magnitudes
across the hybrid-uint split), the mixed DCT32/16/8 layout of
src/entropy_gpu_test.cc:88-111, the DC pattern of
src/dc_entropy_gpu_test.cc:41-54 and the CfL maps of
src/dc_entropy_gpu_test.cc:81-88. Planes use the encoder's layouts: AC
[3][B*64] covered-block slots, DC [3][B], channels X, Y, B.
"""

from __future__ import annotations

import numpy as np


def covered_slot(n: int, bx: int, by: int, bw: int, raw: int) -> int:
    side = n // 8
    q = raw // 64
    return ((by + q // side) * bw + bx + q % side) * 64 + raw % 64


def empty(w: int, h: int, qf: int = 32) -> dict:
    bw, bh = w // 8, h // 8
    nb = bw * bh
    nt = ((bw + 7) // 8) * ((bh + 7) // 8)
    return {"w": w, "h": h, "ac": np.zeros((3, nb * 64), np.int16), "dc": np.zeros((3, nb), np.int32),
            "acs": np.full(nb, 8, np.int8), "qf": np.full(nb, qf, np.int32),
            "ytox": np.zeros(nt, np.int8), "ytob": np.zeros(nt, np.int8)}


def fill_ac_pattern(f: dict) -> None:
    bw, bh = f["w"] // 8, f["h"] // 8
    for by in range(bh):
        for bx in range(bw):
            b = (by * bw + bx) * 64
            for c in range(3):
                blk = f["ac"][c]
                blk[b + 1] = (bx + c) % 7 - 3
                blk[b + 8] = (by * 2 + c) % 11 - 5
                blk[b + 9] = (bx + by) % 5 - 2
                blk[b + 16] = (bx * 3 + by) % 260 - 130
                blk[b + 2] = (by + c) % 3 - 1


def set_first_block(f: dict, side: int, bx: int, by: int) -> None:
    bw = f["w"] // 8
    s = side // 8
    for dy in range(s):
        for dx in range(s):
            f["acs"][(by + dy) * bw + bx + dx] = side if (dx == 0 and dy == 0) else 0


def make_mixed(w: int, h: int) -> dict:
    f = empty(w, h)
    bw, bh = w // 8, h // 8
    set_first_block(f, 32, 0, 0)
    set_first_block(f, 16, 4, 0)
    set_first_block(f, 16, 0, 4)
    for by in range(bh):
        for bx in range(bw):
            n = int(f["acs"][by * bw + bx])
            if n == 0:
                continue
            for raw in range(1, n * n, 3):
                s = covered_slot(n, bx, by, bw, raw)
                for c in range(3):
                    f["ac"][c][s] = (raw + bx + by + c) % 9 - 4
    return f


def fill_dc_pattern(f: dict) -> None:
    bw, bh = f["w"] // 8, f["h"] // 8
    by, bx = np.mgrid[0:bh, 0:bw]
    f["dc"][0] = ((bx * 3 + by) % 517 - 258).ravel()
    f["dc"][1] = ((bx + by * 2) % 41 - 20).ravel()
    f["dc"][2] = ((bx + by) % 7 - 3).ravel()


def fill_cfl_pattern(f: dict) -> None:
    i = np.arange(f["ytox"].size)
    f["ytox"][:] = i % 13 - 6
    f["ytob"][:] = i % 9 - 4


def mixed_full(w: int, h: int, seed: int | None = None) -> dict:
    """Mixed layout with AC, DC and CfL patterns; with a seed, a random per-block
    quant field in [1, 256]."""
    f = make_mixed(w, h)
    fill_dc_pattern(f)
    fill_cfl_pattern(f)
    if seed is not None:
        rng = np.random.Generator(np.random.PCG64(seed))
        f["qf"][:] = rng.integers(1, 257, f["qf"].size)
    return f


def flat(f: dict) -> dict:
    return {"ac": f["ac"].ravel(), "dc": f["dc"].ravel(), "acs": f["acs"], "qf": f["qf"],
            "ytox": f["ytox"], "ytob": f["ytob"]}
