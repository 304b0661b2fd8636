"""Decoding the files this encoder writes, on the host, through the in-tree
subset decoder (csrc/subset_decoder.cc): decodability checks and luma PSNR.

    from cujpegxl_b200.decode import decode, psnr_y
    img = decode(data)             # DecodedImage(width, height, xyb, srgb)
    db = psnr_y(nv12, data)        # PSNR of BT.709 Y' against the input luma
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libjxlsubset.so"
_lib: ctypes.CDLL | None = None


def _load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m cujpegxl_b200.build`")
        L = ctypes.CDLL(str(LIB_PATH))
        L.jxlsubset_decode.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint32),
                                       ctypes.POINTER(ctypes.c_uint32), ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t]
        L.jxlsubset_decode.restype = ctypes.c_int
        U32 = ctypes.POINTER(ctypes.c_uint32)
        L.jxlsubset_decode_planes.argtypes = [ctypes.c_void_p, ctypes.c_size_t, U32, U32] + [ctypes.c_void_p] * 6 + [
            U32, U32, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t]
        L.jxlsubset_decode_planes.restype = ctypes.c_int
        _lib = L
    return _lib


class DecodeError(ValueError):
    pass


@dataclass
class DecodedImage:
    width: int
    height: int
    xyb: np.ndarray    # float32 [3][H][W]
    srgb: np.ndarray   # float32 [3][H][W], in [0, 1]

    def luma(self) -> np.ndarray:
        """BT.709 Y' in [0, 255] (the weights of the encoder's Y'CbCr input)."""
        r, g, b = self.srgb
        return 255.0 * (0.2126 * r + 0.7152 * g + 0.0722 * b)


def decode(data: bytes) -> DecodedImage:
    L = _load()
    buf = np.frombuffer(data, np.uint8)
    w = ctypes.c_uint32(0)
    h = ctypes.c_uint32(0)
    err = ctypes.create_string_buffer(512)
    code = L.jxlsubset_decode(buf.ctypes.data, buf.size, ctypes.byref(w), ctypes.byref(h), None, None, 0, err, 512)
    if code == 1:
        raise DecodeError(err.value.decode())
    p = w.value * h.value
    xyb = np.empty((3, h.value, w.value), np.float32)
    srgb = np.empty((3, h.value, w.value), np.float32)
    code = L.jxlsubset_decode(buf.ctypes.data, buf.size, ctypes.byref(w), ctypes.byref(h), xyb.ctypes.data,
                              srgb.ctypes.data, p, err, 512)
    if code != 0:
        raise DecodeError(err.value.decode())
    return DecodedImage(w.value, h.value, xyb, srgb)


def decode_planes(data: bytes) -> dict:
    """The quantised planes and quantiser state stored in a file (the layouts of
    cujpegxl_b200_planes), for encode -> decode round trips."""
    L = _load()
    buf = np.frombuffer(data, np.uint8)
    w = ctypes.c_uint32(0)
    h = ctypes.c_uint32(0)
    gs = ctypes.c_uint32(0)
    qdc = ctypes.c_uint32(0)
    err = ctypes.create_string_buffer(512)
    args = [None] * 6
    code = L.jxlsubset_decode_planes(buf.ctypes.data, buf.size, ctypes.byref(w), ctypes.byref(h), *args,
                                     ctypes.byref(gs), ctypes.byref(qdc), 0, err, 512)
    if code == 1:
        raise DecodeError(err.value.decode())
    bw, bh = w.value // 8, h.value // 8
    nb, nt = bw * bh, ((bw + 7) // 8) * ((bh + 7) // 8)
    r = {"ac": np.zeros(3 * nb * 64, np.int16), "dc": np.zeros(3 * nb, np.int32), "acs": np.zeros(nb, np.int8),
         "qf": np.zeros(nb, np.int32), "ytox": np.zeros(nt, np.int8), "ytob": np.zeros(nt, np.int8)}
    code = L.jxlsubset_decode_planes(buf.ctypes.data, buf.size, ctypes.byref(w), ctypes.byref(h),
                                     *[r[k].ctypes.data for k in ("ac", "dc", "acs", "qf", "ytox", "ytob")],
                                     ctypes.byref(gs), ctypes.byref(qdc), nb, err, 512)
    if code != 0:
        raise DecodeError(err.value.decode())
    r.update(width=w.value, height=h.value, global_scale=gs.value, quant_dc=qdc.value)
    return r


def psnr_y(nv12: np.ndarray, data: bytes) -> float:
    img = decode(data)
    y = np.asarray(nv12, np.uint8).ravel()[: img.width * img.height].reshape(img.height, img.width)
    mse = float(np.mean((img.luma() - y.astype(np.float64)) ** 2))
    return float("inf") if mse == 0 else 10.0 * np.log10(255.0 ** 2 / mse)
