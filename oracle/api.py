"""ctypes bindings over the CPU restatement (liboracle.so) and the reference
checker library (_ref/libjxlref.so). Test infrastructure only: imported by
tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, and
only as the checker or the timed CPU baseline.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libjxlref.so"

_P = ctypes.c_void_p


def _ptr(a: np.ndarray | None) -> int | None:
    return None if a is None else a.ctypes.data


class _Frame(ctypes.Structure):
    _fields_ = [("luma", _P), ("chroma", _P), ("luma_pitch", ctypes.c_size_t),
                ("chroma_pitch", ctypes.c_size_t), ("width", ctypes.c_int), ("height", ctypes.c_int)]


class _Outputs(ctypes.Structure):
    _fields_ = [(n, _P) for n in ("ac", "dc", "acs", "qf", "ytox", "ytob", "nzn", "nzc",
                                   "dbg_xyb", "dbg_sharp", "dbg_coeff")]


class _Scalars(ctypes.Structure):
    _fields_ = [("global_scale", ctypes.c_uint32), ("quant_dc", ctypes.c_uint32),
                ("raw_quant_field", ctypes.c_uint32), ("gsf", ctypes.c_float),
                ("inv_global_scale", ctypes.c_float), ("qgsf_select", ctypes.c_float),
                ("dc_scale", ctypes.c_float), ("mul_pb", ctypes.c_float), ("add_pb", ctypes.c_float),
                ("km", ctypes.c_float * 4)]


_oracle = None
_ref = None


def oracle() -> ctypes.CDLL:
    global _oracle
    if _oracle is None:
        lib = ctypes.CDLL(str(ORACLE_LIB))
        lib.oracle_frontend.argtypes = [ctypes.POINTER(_Frame), ctypes.c_float, ctypes.POINTER(_Outputs), ctypes.c_int]
        lib.oracle_assemble.restype = ctypes.c_size_t
        lib.oracle_assemble.argtypes = [ctypes.c_int, ctypes.c_int] + [_P] * 6 + [ctypes.c_uint32] * 2 + [_P, ctypes.c_size_t]
        lib.oracle_encode.restype = ctypes.c_size_t
        lib.oracle_encode.argtypes = [ctypes.POINTER(_Frame), ctypes.c_float, _P, ctypes.c_size_t, ctypes.c_int]
        lib.oracle_huffman.restype = ctypes.c_size_t
        lib.oracle_huffman.argtypes = [_P, ctypes.c_size_t, _P, _P, _P, ctypes.c_size_t]
        lib.oracle_scalars.argtypes = [ctypes.c_float, ctypes.POINTER(_Scalars)]
        for name in ("oracle_log2", "oracle_exp2", "oracle_exp", "oracle_cbrt", "oracle_pow24"):
            getattr(lib, name).restype = ctypes.c_float
            getattr(lib, name).argtypes = [ctypes.c_float]
        lib.oracle_f2h.restype = ctypes.c_uint16
        lib.oracle_f2h.argtypes = [ctypes.c_float]
        lib.oracle_ratio_gamma.restype = ctypes.c_float
        lib.oracle_ratio_gamma.argtypes = [ctypes.c_float, ctypes.c_int]
        lib.oracle_masking_sqrt.restype = ctypes.c_float
        lib.oracle_masking_sqrt.argtypes = [ctypes.c_float]
        lib.oracle_compute_mask.restype = ctypes.c_float
        lib.oracle_compute_mask.argtypes = [ctypes.c_float]
        lib.oracle_gaborish_weights.argtypes = [_P]
        lib.oracle_sel_cost.restype = ctypes.c_float
        lib.oracle_sel_cost.argtypes = [_P, ctypes.c_int, ctypes.c_int, ctypes.c_float]
        lib.oracle_select_plane.argtypes = [_P, ctypes.c_int, ctypes.c_int, ctypes.c_float, _P]
        lib.oracle_dc_from_llf.argtypes = [ctypes.c_int, _P, _P]
        lib.oracle_cfl_maps.argtypes = [ctypes.c_float] * 3 + [_P, _P]
        lib.oracle_xyb_pixel.argtypes = [ctypes.POINTER(_Frame), ctypes.c_int, ctypes.c_int, _P]
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return REF_LIB.exists()


def ref() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        lib = ctypes.CDLL(str(REF_LIB))
        lib.ref_select_transforms.argtypes = [_P, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_float, _P]
        lib.ref_block_ac_cost.restype = ctypes.c_float
        lib.ref_block_ac_cost.argtypes = [_P, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int, ctypes.c_float]
        lib.ref_huffman.restype = ctypes.c_size_t
        lib.ref_huffman.argtypes = [_P, ctypes.c_size_t, _P, _P, _P, ctypes.c_size_t]
        lib.ref_encode_frame.restype = ctypes.c_size_t
        lib.ref_encode_frame.argtypes = [ctypes.c_size_t, ctypes.c_size_t] + [_P] * 6 + [ctypes.c_uint32] * 2 + [_P, ctypes.c_size_t]
        lib.ref_write_codestream.restype = ctypes.c_size_t
        lib.ref_write_codestream.argtypes = [ctypes.c_size_t, ctypes.c_size_t] + [_P] * 5 + [ctypes.c_uint32] * 3 + [_P, ctypes.c_size_t]
        lib.ref_ac_encode.restype = ctypes.c_size_t
        lib.ref_ac_encode.argtypes = [ctypes.c_size_t, ctypes.c_size_t, _P, _P, _P, _P, _P, _P, ctypes.c_size_t, _P]
        lib.ref_dc_encode.restype = ctypes.c_size_t
        lib.ref_dc_encode.argtypes = [ctypes.c_size_t, ctypes.c_size_t, _P, _P, _P, _P, ctypes.c_uint32, _P, ctypes.c_size_t, _P, _P, _P]
        lib.ref_xyb_pixel.argtypes = [ctypes.c_float] * 3 + [_P] * 3
        lib.ref_xyb_constants.argtypes = [_P]
        lib.ref_gaborish_weights.argtypes = [_P]
        for name in ("ref_masking_sqrt", "ref_compute_mask"):
            getattr(lib, name).restype = ctypes.c_float
            getattr(lib, name).argtypes = [ctypes.c_float]
        lib.ref_ratio_cbrt_gamma.restype = ctypes.c_float
        lib.ref_ratio_cbrt_gamma.argtypes = [ctypes.c_float, ctypes.c_int]
        lib.ref_calibrate.argtypes = [ctypes.c_float, _P, _P]
        lib.ref_natural_order.argtypes = [ctypes.c_int, _P]
        lib.ref_dequant_weights.argtypes = [ctypes.c_int, ctypes.c_int, _P]
        lib.ref_dc_from_llf.argtypes = [ctypes.c_int, _P, _P]
        lib.ref_cfl_maps_from_sums.argtypes = [ctypes.c_double] * 3 + [_P, _P]
        lib.ref_ac_cluster.argtypes = [ctypes.c_uint32]
        lib.ref_ac_zero_density_context.restype = ctypes.c_uint32
        lib.ref_ac_zero_density_context.argtypes = [ctypes.c_uint32] * 5
        lib.ref_ac_nonzero_context.restype = ctypes.c_uint32
        lib.ref_ac_nonzero_context.argtypes = [ctypes.c_uint32, ctypes.c_int]
        lib.ref_gradient_predict.restype = ctypes.c_int32
        lib.ref_gradient_predict.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
        _ref = lib
    return _ref


def split_nv12(nv12: np.ndarray, width: int, height: int) -> tuple[np.ndarray, np.ndarray]:
    flat = np.ascontiguousarray(nv12, dtype=np.uint8).ravel()
    return flat[: width * height], flat[width * height: width * height * 3 // 2]


class FrontendResult:
    """Planes produced by the frontend (CPU restatement or CUDA)."""

    def __init__(self, width: int, height: int, debug: bool = False):
        bw, bh = width // 8, height // 8
        nb = bw * bh
        nt = ((bw + 7) // 8) * ((bh + 7) // 8)
        self.width, self.height = width, height
        self.ac = np.zeros(3 * nb * 64, np.int16)
        self.dc = np.zeros(3 * nb, np.int32)
        self.acs = np.zeros(nb, np.int8)
        self.qf = np.zeros(nb, np.int32)
        self.ytox = np.zeros(nt, np.int8)
        self.ytob = np.zeros(nt, np.int8)
        self.nzn = np.zeros(3 * nb, np.uint8)
        self.nzc = np.zeros(3 * nb, np.uint16)
        self.xyb = np.zeros(3 * width * height, np.float32) if debug else None
        self.sharp = np.zeros(3 * width * height, np.float32) if debug else None
        self.coeff = np.zeros(3 * nb * 64, np.uint16) if debug else None


def scalars(distance: float) -> dict:
    s = _Scalars()
    oracle().oracle_scalars(distance, ctypes.byref(s))
    return {"global_scale": s.global_scale, "quant_dc": s.quant_dc, "raw_quant_field": s.raw_quant_field,
            "gsf": s.gsf, "inv_global_scale": s.inv_global_scale, "qgsf_select": s.qgsf_select,
            "dc_scale": s.dc_scale}


def frontend(nv12: np.ndarray, width: int, height: int, distance: float, debug: bool = False,
             threads: int | None = None) -> FrontendResult:
    luma, chroma = split_nv12(nv12, width, height)
    fr = _Frame(luma.ctypes.data, chroma.ctypes.data, width, width, width, height)
    r = FrontendResult(width, height, debug)
    o = _Outputs(*[_ptr(a) for a in (r.ac, r.dc, r.acs, r.qf, r.ytox, r.ytob, r.nzn, r.nzc,
                                     r.xyb, r.sharp, r.coeff)])
    n = threads if threads is not None else (os.cpu_count() or 1)
    if oracle().oracle_frontend(ctypes.byref(fr), distance, ctypes.byref(o), n) != 0:
        raise ValueError("oracle_frontend rejected the frame")
    return r


def assemble(r: FrontendResult, distance: float) -> bytes:
    s = scalars(distance)
    cap = max(3 * r.acs.size * 384 + 48 * r.acs.size + (1 << 16), 1 << 20)
    out = np.zeros(cap, np.uint8)
    n = oracle().oracle_assemble(r.width, r.height, _ptr(r.ac), _ptr(r.dc), _ptr(r.acs), _ptr(r.qf),
                                 _ptr(r.ytox), _ptr(r.ytob), s["global_scale"], s["quant_dc"],
                                 _ptr(out), cap)
    return out[:n].tobytes()


def encode(nv12: np.ndarray, width: int, height: int, distance: float, threads: int | None = None) -> bytes:
    luma, chroma = split_nv12(nv12, width, height)
    fr = _Frame(luma.ctypes.data, chroma.ctypes.data, width, width, width, height)
    bw, bh = width // 8, height // 8
    cap = max(3 * bw * bh * 384 + (1 << 20), 1 << 20)
    out = np.zeros(cap, np.uint8)
    n = threads if threads is not None else (os.cpu_count() or 1)
    size = oracle().oracle_encode(ctypes.byref(fr), distance, _ptr(out), cap, n)
    return out[:size].tobytes()


def ref_encode_frame(r: FrontendResult, distance: float) -> bytes:
    s = scalars(distance)
    ac32 = r.ac.astype(np.int32)
    cap = max(3 * r.acs.size * 384 + (1 << 20), 1 << 20)
    out = np.zeros(cap, np.uint8)
    n = ref().ref_encode_frame(r.width, r.height, _ptr(ac32), _ptr(r.dc), _ptr(r.acs), _ptr(r.ytox),
                               _ptr(r.ytob), _ptr(r.qf), s["global_scale"], s["quant_dc"], _ptr(out), cap)
    return out[:n].tobytes()


def ref_select(sharp_y: np.ndarray, width: int, height: int, distance: float) -> np.ndarray:
    acs = np.full((width // 8) * (height // 8), -1, np.int8)
    y = np.ascontiguousarray(sharp_y, np.float32)
    ref().ref_select_transforms(_ptr(y), width, height, distance, _ptr(acs))
    return acs
