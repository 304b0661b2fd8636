"""The device prefix-code builder (the warp-cooperative construction every
encode runs: one merge per count floor on every lane, canonical codes and the
code-length-code header written across the warp) against the reference's
own build_and_store_huffman_tree outputs in tests/golden/huffman.npz: 27
histograms from one to 256 symbols, Fibonacci counts that force the 15-bit
depth limit, sparse and dense random cases. Depths, codes, header bits and
header length must all be equal."""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np
import pytest

from cujpegxl_b200 import _capi

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden" / "huffman.npz"


def test_device_prefix_codes_equal_reference_golden():
    z = np.load(GOLD)
    L = _capi.lib()
    i = 0
    limited = 0
    while f"hist{i}" in z:
        h = np.ascontiguousarray(z[f"hist{i}"].astype(np.uint32))
        depth = np.zeros(h.size, np.uint8)
        bits = np.zeros(h.size, np.uint16)
        head = np.zeros(256, np.uint8)
        nbits = ctypes.c_uint32(0)
        code = L.cujpegxl_b200_debug_prefix_code(0, h.ctypes.data, h.size, depth.ctypes.data, bits.ctypes.data,
                                                 head.ctypes.data, head.size, ctypes.byref(nbits))
        assert code == _capi.OK, i
        np.testing.assert_array_equal(depth, z[f"depth{i}"], err_msg=f"case {i}")
        np.testing.assert_array_equal(bits, z[f"bits{i}"], err_msg=f"case {i}")
        assert nbits.value == int(z[f"nbits{i}"][0]), i
        np.testing.assert_array_equal(head[: (nbits.value + 7) // 8], z[f"header{i}"], err_msg=f"case {i}")
        limited += int(depth.max() == 15)
        i += 1
    assert i > 20 and limited >= 1
