"""ctypes binding of libcujpegxl.so.1 (the in-tree CUDA build).

Loading fails loudly when the library has not been built: there is no CPU
fallback anywhere in the package.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libcujpegxl.so.1"

OK = 0
NOT_IMPLEMENTED = 1
INVALID_ARGUMENT = 2
UNSUPPORTED_RESOLUTION = 3
NO_DEVICE = 4
INTERNAL_ERROR = 5
BUFFER_TOO_SMALL = 6

# cujpegxl_b200_encoder_enqueue_stages stage bits.
STAGE_FRONTEND = 1
STAGE_ENTROPY = 2

EXPORTS = (
    "cujpegxl_api_version", "cujpegxl_status_string", "cujpegxl_backend_string",
    "cujpegxl_query_backend", "cujpegxl_max_output_size", "cujpegxl_encoder_create",
    "cujpegxl_encoder_configure", "cujpegxl_encoder_encode", "cujpegxl_encoder_destroy",
    "cujpegxl_b200_encoder_set_debug", "cujpegxl_b200_encoder_read_planes",
    "cujpegxl_b200_encode_planes", "cujpegxl_b200_encode_host", "cujpegxl_b200_encoder_enqueue",
    "cujpegxl_b200_encoder_enqueue_stages", "cujpegxl_b200_encoder_result", "cujpegxl_b200_encoder_stream",
    "cujpegxl_b200_kernels_per_encode", "cujpegxl_b200_encode_planes_noalloc",
    "cujpegxl_b200_batch_create", "cujpegxl_b200_batch_encode", "cujpegxl_b200_batch_sync",
    "cujpegxl_b200_batch_frame", "cujpegxl_b200_batch_copy", "cujpegxl_b200_batch_lanes",
    "cujpegxl_b200_batch_destroy", "cujpegxl_b200_batch_stream", "cujpegxl_b200_encoder_memory",
    "cujpegxl_b200_acsnet_param_count", "cujpegxl_b200_acsnet_check_blob", "cujpegxl_b200_acsnet_create",
    "cujpegxl_b200_acsnet_destroy", "cujpegxl_b200_encoder_set_acsnet", "cujpegxl_b200_encoder_acsnet_stats",
    "cujpegxl_b200_acsnet_trainer_create", "cujpegxl_b200_acsnet_trainer_destroy",
    "cujpegxl_b200_acsnet_trainer_forward", "cujpegxl_b200_acsnet_trainer_gradient",
    "cujpegxl_b200_acsnet_trainer_step", "cujpegxl_b200_acsnet_trainer_params", "cujpegxl_b200_batch_set_acsnet",
    "cujpegxl_b200_encoder_create_ex", "cujpegxl_b200_max_output_size_ex",
    "cujpegxl_b200_debug_fail_allocation", "cujpegxl_b200_debug_live_allocations",
    "cujpegxl_b200_encoder_enqueue_readback", "cujpegxl_b200_batch_schedule",
    "cujpegxl_b200_debug_prefix_code",
)


class Config(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("distance", ctypes.c_float), ("device_ordinal", ctypes.c_int32)]


class Nv12Input(ctypes.Structure):
    _fields_ = [("luma", ctypes.c_size_t), ("chroma", ctypes.c_size_t),
                ("luma_pitch", ctypes.c_size_t), ("chroma_pitch", ctypes.c_size_t)]


class Output(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("size", ctypes.c_size_t), ("capacity", ctypes.c_size_t)]


class Planes(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("ac", "dc", "acs", "qf", "ytox", "ytob", "xyb", "sharp", "coeff",
                                                "cost")]


class NetBatch(ctypes.Structure):
    _fields_ = [("tiles", ctypes.c_size_t), ("tile_index", ctypes.c_size_t), ("log2_distance", ctypes.c_size_t),
                ("label_class", ctypes.c_size_t), ("label_qf", ctypes.c_size_t), ("n", ctypes.c_uint32),
                ("label_soft", ctypes.c_size_t)]


class BatchSchedule(ctypes.Structure):
    _fields_ = [("frontend_ctas", ctypes.c_uint32), ("tiles_per_claim", ctypes.c_uint32),
                ("dynamic_claims", ctypes.c_uint32), ("largest_first", ctypes.c_uint32),
                ("from_cache", ctypes.c_uint32), ("candidates", ctypes.c_uint32), ("tuned_ms", ctypes.c_float),
                ("tiles_per_cta", ctypes.c_uint32)]


class DevicePlanes(ctypes.Structure):
    _fields_ = [(n, ctypes.c_size_t) for n in ("ac", "dc", "acs", "qf", "ytox", "ytob")]


_lib: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m cujpegxl_b200.build`")
    L = ctypes.CDLL(str(LIB_PATH))
    E = ctypes.c_void_p
    P = ctypes.POINTER
    L.cujpegxl_api_version.restype = ctypes.c_uint32
    L.cujpegxl_status_string.restype = ctypes.c_char_p
    L.cujpegxl_status_string.argtypes = [ctypes.c_int]
    L.cujpegxl_backend_string.restype = ctypes.c_char_p
    L.cujpegxl_backend_string.argtypes = [ctypes.c_int]
    L.cujpegxl_query_backend.argtypes = [ctypes.c_int32, P(ctypes.c_int)]
    L.cujpegxl_max_output_size.argtypes = [P(Config), P(ctypes.c_size_t)]
    L.cujpegxl_encoder_create.argtypes = [P(Config), P(E)]
    L.cujpegxl_encoder_configure.argtypes = [E, P(Config)]
    L.cujpegxl_encoder_encode.argtypes = [E, P(Nv12Input), P(Output)]
    L.cujpegxl_encoder_destroy.argtypes = [E]
    L.cujpegxl_encoder_destroy.restype = None
    L.cujpegxl_b200_encoder_set_debug.argtypes = [E, ctypes.c_int32]
    L.cujpegxl_b200_encoder_read_planes.argtypes = [E, P(Planes)]
    L.cujpegxl_b200_encode_planes.argtypes = [E, P(Planes), ctypes.c_uint32, ctypes.c_uint32, P(Output)]
    L.cujpegxl_b200_encode_host.argtypes = [E, ctypes.c_void_p, ctypes.c_size_t, P(Output)]
    L.cujpegxl_b200_encoder_enqueue.argtypes = [E, P(Nv12Input)]
    L.cujpegxl_b200_encoder_enqueue_stages.argtypes = [E, P(Nv12Input), ctypes.c_uint32]
    L.cujpegxl_b200_encoder_result.argtypes = [E, P(ctypes.c_size_t), P(ctypes.c_size_t)]
    L.cujpegxl_b200_encoder_stream.argtypes = [E, P(ctypes.c_size_t)]
    L.cujpegxl_b200_kernels_per_encode.restype = ctypes.c_uint32
    L.cujpegxl_b200_encoder_enqueue_readback.argtypes = [E, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    L.cujpegxl_b200_batch_schedule.argtypes = [E, P(BatchSchedule)]
    L.cujpegxl_b200_debug_prefix_code.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                                  P(ctypes.c_uint32)]
    L.cujpegxl_b200_debug_fail_allocation.argtypes = [ctypes.c_uint32]
    L.cujpegxl_b200_debug_fail_allocation.restype = None
    L.cujpegxl_b200_debug_live_allocations.restype = ctypes.c_uint64
    L.cujpegxl_b200_encoder_memory.argtypes = [E, P(ctypes.c_size_t), P(ctypes.c_size_t)]
    L.cujpegxl_b200_encode_planes_noalloc.argtypes = [P(DevicePlanes), ctypes.c_uint32, ctypes.c_uint32,
                                                      ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p,
                                                      ctypes.c_size_t, P(ctypes.c_size_t), ctypes.c_size_t]
    L.cujpegxl_b200_encode_planes_noalloc.restype = ctypes.c_int
    L.cujpegxl_b200_batch_create.argtypes = [P(Config), ctypes.c_size_t, P(E)]
    L.cujpegxl_b200_batch_encode.argtypes = [E, P(Nv12Input)]
    L.cujpegxl_b200_batch_sync.argtypes = [E, P(ctypes.c_size_t)]
    L.cujpegxl_b200_batch_frame.argtypes = [E, ctypes.c_size_t, P(ctypes.c_size_t), P(ctypes.c_size_t)]
    L.cujpegxl_b200_batch_copy.argtypes = [E, ctypes.c_size_t, P(Output)]
    L.cujpegxl_b200_batch_stream.argtypes = [E, P(ctypes.c_size_t)]
    L.cujpegxl_b200_batch_lanes.argtypes = [E]
    L.cujpegxl_b200_batch_lanes.restype = ctypes.c_uint32
    L.cujpegxl_b200_batch_destroy.argtypes = [E]
    L.cujpegxl_b200_batch_destroy.restype = None
    F = ctypes.c_float
    L.cujpegxl_b200_acsnet_param_count.restype = ctypes.c_uint32
    L.cujpegxl_b200_acsnet_check_blob.argtypes = [ctypes.c_void_p, ctypes.c_size_t]
    L.cujpegxl_b200_acsnet_create.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32, P(E)]
    L.cujpegxl_b200_acsnet_destroy.argtypes = [E]
    L.cujpegxl_b200_acsnet_destroy.restype = None
    L.cujpegxl_b200_encoder_set_acsnet.argtypes = [E, E, F, ctypes.c_uint32]
    L.cujpegxl_b200_encoder_acsnet_stats.argtypes = [E, P(ctypes.c_uint32), P(ctypes.c_uint32)]
    L.cujpegxl_b200_acsnet_trainer_create.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                                      ctypes.c_int32, P(E)]
    L.cujpegxl_b200_acsnet_trainer_destroy.argtypes = [E]
    L.cujpegxl_b200_acsnet_trainer_destroy.restype = None
    L.cujpegxl_b200_acsnet_trainer_forward.argtypes = [E, P(NetBatch), ctypes.c_size_t, ctypes.c_size_t]
    L.cujpegxl_b200_acsnet_trainer_gradient.argtypes = [E, P(NetBatch), F, ctypes.c_size_t, ctypes.c_size_t,
                                                        ctypes.c_size_t]
    L.cujpegxl_b200_acsnet_trainer_step.argtypes = [E, P(NetBatch), F, F, ctypes.c_size_t, ctypes.c_size_t]
    L.cujpegxl_b200_acsnet_trainer_params.argtypes = [E, ctypes.c_void_p]
    L.cujpegxl_b200_batch_set_acsnet.argtypes = [E, E, F, ctypes.c_uint32]
    L.cujpegxl_b200_encoder_create_ex.argtypes = [P(Config), ctypes.c_uint32, P(E)]
    L.cujpegxl_b200_max_output_size_ex.argtypes = [P(Config), ctypes.c_uint32, P(ctypes.c_size_t)]
    for name in ("cujpegxl_query_backend", "cujpegxl_max_output_size", "cujpegxl_encoder_create",
                 "cujpegxl_encoder_configure", "cujpegxl_encoder_encode", "cujpegxl_b200_encoder_set_debug",
                 "cujpegxl_b200_encoder_read_planes", "cujpegxl_b200_encode_planes",
                 "cujpegxl_b200_encode_host", "cujpegxl_b200_encoder_enqueue", "cujpegxl_b200_encoder_enqueue_stages",
                 "cujpegxl_b200_encoder_result", "cujpegxl_b200_encoder_stream", "cujpegxl_b200_batch_create",
                 "cujpegxl_b200_batch_encode", "cujpegxl_b200_batch_sync", "cujpegxl_b200_batch_frame",
                 "cujpegxl_b200_batch_copy", "cujpegxl_b200_batch_stream", "cujpegxl_b200_encoder_memory",
                 "cujpegxl_b200_acsnet_check_blob", "cujpegxl_b200_acsnet_create", "cujpegxl_b200_encoder_set_acsnet",
                 "cujpegxl_b200_encoder_acsnet_stats", "cujpegxl_b200_acsnet_trainer_create",
                 "cujpegxl_b200_acsnet_trainer_forward", "cujpegxl_b200_acsnet_trainer_gradient",
                 "cujpegxl_b200_acsnet_trainer_step", "cujpegxl_b200_acsnet_trainer_params",
                 "cujpegxl_b200_batch_set_acsnet", "cujpegxl_b200_encoder_create_ex",
                 "cujpegxl_b200_max_output_size_ex"):
        getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


def status_string(code: int) -> str:
    return lib().cujpegxl_status_string(code).decode()


class CujpegxlError(RuntimeError):
    def __init__(self, what: str, code: int):
        super().__init__(f"{what} failed: {status_string(code)}")
        self.code = code


def check(what: str, code: int) -> None:
    if code != OK:
        raise CujpegxlError(what, code)


def ptr(a: np.ndarray | None) -> int | None:
    return None if a is None else a.ctypes.data
