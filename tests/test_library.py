"""The C-ABI library without a GPU: it loads, exports exactly the symbols the
headers declare, and applies the reference's argument checks and output
bound (src/cujpegxl.cc:36-59, 69-88) before touching a device."""

from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import cujpegxl_b200 as cj
from cujpegxl_b200 import _capi

REPO = Path(__file__).resolve().parents[1]


def declared_symbols() -> set[str]:
    names = set()
    for h in (REPO / "include").rglob("*.h"):
        names |= set(re.findall(r"\b(cujpegxl_\w+)\s*\(", h.read_text()))
    return names


def test_exports_match_headers():
    out = subprocess.run(["nm", "-D", "--defined-only", str(_capi.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {m.group(1) for m in re.finditer(r" T (cujpegxl_\w+)@@CUJPEGXL_1", out)}
    assert exported == declared_symbols()
    assert set(_capi.EXPORTS) == exported
    others = [l for l in out.splitlines() if " T " in l and "cujpegxl_" not in l]
    assert others == []


def test_soname_and_reference_symbols():
    out = subprocess.run(["readelf", "-d", str(_capi.LIB_PATH)], capture_output=True, text=True).stdout
    assert "libcujpegxl.so.1" in out
    ref = {"cujpegxl_api_version", "cujpegxl_status_string", "cujpegxl_backend_string", "cujpegxl_query_backend",
           "cujpegxl_max_output_size", "cujpegxl_encoder_create", "cujpegxl_encoder_configure",
           "cujpegxl_encoder_encode", "cujpegxl_encoder_destroy"}
    assert ref <= declared_symbols()


def test_strings_and_version():
    L = _capi.lib()
    assert L.cujpegxl_api_version() == 3 == cj.API_VERSION == cj.api_version()
    names = ["ok", "not-implemented", "invalid-argument", "unsupported-resolution", "no-device",
             "internal-error", "buffer-too-small"]
    assert [_capi.status_string(i) for i in range(7)] == names
    assert _capi.status_string(99) == "internal-error"
    assert [L.cujpegxl_backend_string(i).decode() for i in range(3)] == ["unknown", "fp32-simt", "fp16-tensor"]


def _bound(w, h):
    bw, bh = w // 8, h // 8
    nac = ((bw + 31) // 32) * ((bh + 31) // 32)
    ndc = ((bw + 255) // 256) * ((bh + 255) // 256)
    return 3 * bw * bh * 384 + 48 * bw * bh + (nac + ndc) * 2048 + 16384


@pytest.mark.parametrize("w,h", [(3840, 2160), (1920, 1080), (264, 8), (4096, 2160), (512, 384)])
def test_max_output_size(w, h):
    assert cj.max_output_size(w, h) == _bound(w, h)


@pytest.mark.parametrize("cfg,code", [
    ((3840, 2160, 0.0, 0), _capi.INVALID_ARGUMENT),
    ((3840, 2160, -1.0, 0), _capi.INVALID_ARGUMENT),
    ((3840, 2160, float("nan"), 0), _capi.INVALID_ARGUMENT),
    ((3840, 2160, float("inf"), 0), _capi.INVALID_ARGUMENT),
    ((100, 100, 1.0, 0), _capi.UNSUPPORTED_RESOLUTION),
    ((256, 256, 1.0, 0), _capi.UNSUPPORTED_RESOLUTION),   # one AC group
    ((0, 512, 1.0, 0), _capi.UNSUPPORTED_RESOLUTION),
    ((516, 512, 1.0, 0), _capi.UNSUPPORTED_RESOLUTION),
    ((512, 500, 1.0, 0), _capi.UNSUPPORTED_RESOLUTION),
])
def test_config_validation(cfg, code):
    L = _capi.lib()
    c = _capi.Config(*cfg)
    out = ctypes.c_size_t(7)
    assert L.cujpegxl_max_output_size(ctypes.byref(c), ctypes.byref(out)) == code
    h = ctypes.c_void_p(123)
    assert L.cujpegxl_encoder_create(ctypes.byref(c), ctypes.byref(h)) == code
    assert h.value is None


def test_null_arguments():
    L = _capi.lib()
    c = _capi.Config(512, 512, 1.0, 0)
    out = ctypes.c_size_t(0)
    assert L.cujpegxl_max_output_size(None, ctypes.byref(out)) == _capi.INVALID_ARGUMENT
    assert L.cujpegxl_max_output_size(ctypes.byref(c), None) == _capi.INVALID_ARGUMENT
    assert L.cujpegxl_encoder_create(None, None) == _capi.INVALID_ARGUMENT
    assert L.cujpegxl_encoder_configure(None, ctypes.byref(c)) == _capi.INVALID_ARGUMENT
    assert L.cujpegxl_encoder_encode(None, None, None) == _capi.INVALID_ARGUMENT
    assert L.cujpegxl_query_backend(0, None) == _capi.INVALID_ARGUMENT
    L.cujpegxl_encoder_destroy(None)


def _has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_no_device_reported():
    L = _capi.lib()
    c = _capi.Config(512, 512, 1.0, 0)
    h = ctypes.c_void_p(None)
    assert L.cujpegxl_encoder_create(ctypes.byref(c), ctypes.byref(h)) == _capi.NO_DEVICE
    b = ctypes.c_int(0)
    assert L.cujpegxl_query_backend(0, ctypes.byref(b)) == _capi.NO_DEVICE
    c.device_ordinal = -1
    assert L.cujpegxl_encoder_create(ctypes.byref(c), ctypes.byref(h)) == _capi.NO_DEVICE


def test_python_mirror_rejects_bad_arrays():
    with pytest.raises(ValueError):
        cj.encode(np.zeros(100, np.uint8), 512, 512)
    with pytest.raises(ValueError):
        cj.encode(np.zeros(512 * 512 * 3 // 2, np.int16), 512, 512)
    with pytest.raises(ValueError):
        cj.encode(np.zeros((512 * 3 // 2, 2 * 512), np.uint8)[:, ::2], 512, 512)
