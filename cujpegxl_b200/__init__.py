"""B200 JPEG XL VarDCT encoder: Python host interface.

Mirrors the reference's Python module `pycujpegxl` (python/pycujpegxl.cc:81-90
in m-pilia/cujpegxl): `API_VERSION`, `api_version()`, `query_backend()`,
`encode(nv12, width, height, distance=1.0, device_ordinal=0) -> bytes` and
`encode_with_stats(...) -> (bytes, [stage records])`, with the same argument
meaning and the same errors (ValueError for a malformed array, RuntimeError for
a failed encode). Every call goes through the C ABI of the in-tree
libcujpegxl.so.1; nothing falls back to the CPU.

`Encoder` exposes the full C ABI, including device-resident inputs and the
stage-level entry points.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _capi
from ._capi import CujpegxlError, check

__all__ = ["API_VERSION", "api_version", "query_backend", "encode", "encode_with_stats", "Encoder", "Batch",
           "CujpegxlError", "max_output_size"]


def api_version() -> int:
    return int(_capi.lib().cujpegxl_api_version())


API_VERSION = 3


def query_backend(device_ordinal: int = 0) -> str:
    L = _capi.lib()
    out = ctypes.c_int(0)
    code = L.cujpegxl_query_backend(device_ordinal, ctypes.byref(out))
    if code != _capi.OK:
        raise RuntimeError("query_backend failed: " + _capi.status_string(code))
    return L.cujpegxl_backend_string(out.value).decode()


SINGLE_GROUP = 1  # CUJPEGXL_B200_ENCODER_SINGLE_GROUP


def max_output_size(width: int, height: int, distance: float = 1.0, device_ordinal: int = 0,
                    flags: int = 0) -> int:
    cfg = _capi.Config(width, height, distance, device_ordinal)
    out = ctypes.c_size_t(0)
    check("max_output_size", _capi.lib().cujpegxl_b200_max_output_size_ex(ctypes.byref(cfg), flags,
                                                                          ctypes.byref(out)))
    return out.value


class Encoder:
    """One encoder handle (cujpegxl_encoder_create ... _destroy).
    flags=SINGLE_GROUP also accepts frames of one 256x256 AC group
    (cujpegxl_b200_encoder_create_ex)."""

    def __init__(self, width: int, height: int, distance: float = 1.0, device_ordinal: int = 0, flags: int = 0):
        self._L = _capi.lib()
        self._h = ctypes.c_void_p(None)
        cfg = _capi.Config(width, height, distance, device_ordinal)
        check("encoder_create", self._L.cujpegxl_b200_encoder_create_ex(ctypes.byref(cfg), flags,
                                                                        ctypes.byref(self._h)))
        self.width, self.height, self.distance, self.device_ordinal = width, height, distance, device_ordinal
        self.flags = flags
        self._buf = np.zeros(max_output_size(width, height, distance, device_ordinal, flags), np.uint8)
        self._net = None

    def close(self) -> None:
        if self._h:
            self._L.cujpegxl_encoder_destroy(self._h)
            self._h = ctypes.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def configure(self, width: int, height: int, distance: float, device_ordinal: int | None = None) -> None:
        dev = self.device_ordinal if device_ordinal is None else device_ordinal
        cfg = _capi.Config(width, height, distance, dev)
        check("encoder_configure", self._L.cujpegxl_encoder_configure(self._h, ctypes.byref(cfg)))
        self.width, self.height, self.distance, self.device_ordinal = width, height, distance, dev
        self._buf = np.zeros(max_output_size(width, height, distance, dev, self.flags), np.uint8)

    def _output(self, capacity: int | None = None) -> _capi.Output:
        cap = self._buf.size if capacity is None else capacity
        return _capi.Output(self._buf.ctypes.data, 0, cap)

    def encode_device(self, luma: int, chroma: int, luma_pitch: int, chroma_pitch: int,
                      capacity: int | None = None) -> bytes:
        """cujpegxl_encoder_encode on device NV12 planes given as addresses."""
        inp = _capi.Nv12Input(luma, chroma, luma_pitch, chroma_pitch)
        out = self._output(capacity)
        check("encoder_encode", self._L.cujpegxl_encoder_encode(self._h, ctypes.byref(inp), ctypes.byref(out)))
        return self._buf[:out.size].tobytes()

    def encode_device_into(self, luma: int, chroma: int, luma_pitch: int, chroma_pitch: int,
                           out_address: int, capacity: int) -> int:
        """cujpegxl_encoder_encode writing into caller host memory; returns the size."""
        inp = _capi.Nv12Input(luma, chroma, luma_pitch, chroma_pitch)
        out = _capi.Output(out_address, 0, capacity)
        check("encoder_encode", self._L.cujpegxl_encoder_encode(self._h, ctypes.byref(inp), ctypes.byref(out)))
        return out.size

    def enqueue_stages(self, luma: int, chroma: int, luma_pitch: int, chroma_pitch: int, stages: int) -> None:
        inp = _capi.Nv12Input(luma, chroma, luma_pitch, chroma_pitch)
        check("encoder_enqueue_stages",
              self._L.cujpegxl_b200_encoder_enqueue_stages(self._h, ctypes.byref(inp), stages))

    def encode_host(self, nv12: np.ndarray) -> bytes:
        a = np.ascontiguousarray(nv12, dtype=np.uint8)
        out = self._output()
        check("encode_host", self._L.cujpegxl_b200_encode_host(self._h, a.ctypes.data, a.size, ctypes.byref(out)))
        return self._buf[:out.size].tobytes()

    def set_debug(self, enable: bool) -> None:
        check("set_debug", self._L.cujpegxl_b200_encoder_set_debug(self._h, 1 if enable else 0))

    def read_planes(self, debug: bool = False, keys=None) -> dict:
        """Planes of the last encode (the stage dumps too with debug=True);
        `keys` restricts the copy to the named planes."""
        bw, bh = self.width // 8, self.height // 8
        nb, nt = bw * bh, ((bw + 7) // 8) * ((bh + 7) // 8)
        shapes = {"ac": (3 * nb * 64, np.int16), "dc": (3 * nb, np.int32), "acs": (nb, np.int8),
                  "qf": (nb, np.int32), "ytox": (nt, np.int8), "ytob": (nt, np.int8)}
        if debug:
            shapes.update({"xyb": (3 * self.width * self.height, np.float32),
                           "sharp": (3 * self.width * self.height, np.float32),
                           "coeff": (3 * nb * 64, np.uint16), "cost": (3 * nb, np.float32)})
        r = {k: np.zeros(n, dt) for k, (n, dt) in shapes.items() if keys is None or k in keys}
        p = _capi.Planes(*[_capi.ptr(r.get(k)) for k in ("ac", "dc", "acs", "qf", "ytox", "ytob",
                                                         "xyb", "sharp", "coeff", "cost")])
        check("read_planes", self._L.cujpegxl_b200_encoder_read_planes(self._h, ctypes.byref(p)))
        return r

    def encode_planes(self, planes: dict, global_scale: int, quant_dc: int) -> bytes:
        keep = {k: np.ascontiguousarray(planes[k], dt) for k, dt in
                (("ac", np.int16), ("dc", np.int32), ("acs", np.int8), ("qf", np.int32),
                 ("ytox", np.int8), ("ytob", np.int8))}
        p = _capi.Planes(*[_capi.ptr(keep.get(k)) for k in ("ac", "dc", "acs", "qf", "ytox", "ytob")],
                         None, None, None, None)
        out = self._output()
        check("encode_planes", self._L.cujpegxl_b200_encode_planes(self._h, ctypes.byref(p), global_scale,
                                                                   quant_dc, ctypes.byref(out)))
        return self._buf[:out.size].tobytes()

    def enqueue(self, luma: int, chroma: int, luma_pitch: int, chroma_pitch: int) -> None:
        inp = _capi.Nv12Input(luma, chroma, luma_pitch, chroma_pitch)
        check("encoder_enqueue", self._L.cujpegxl_b200_encoder_enqueue(self._h, ctypes.byref(inp)))

    def result(self) -> tuple[int, int]:
        size = ctypes.c_size_t(0)
        dev = ctypes.c_size_t(0)
        check("encoder_result", self._L.cujpegxl_b200_encoder_result(self._h, ctypes.byref(size), ctypes.byref(dev)))
        return size.value, dev.value

    def stream(self) -> int:
        s = ctypes.c_size_t(0)
        check("encoder_stream", self._L.cujpegxl_b200_encoder_stream(self._h, ctypes.byref(s)))
        return s.value

    def set_acsnet(self, net, margin: float = 0.2, flags: int = 1) -> None:
        """Attach a transform-decision network (cujpegxl_b200.acsnet.AcsNet;
        None detaches). flags: 1 = split only, 3 = split and quant field."""
        check("encoder_set_acsnet", self._L.cujpegxl_b200_encoder_set_acsnet(
            self._h, None if net is None else net.handle, margin, flags))
        self._net = net

    def acsnet_stats(self) -> tuple[int, int]:
        """(regions the network decided, full 32x32 regions) of the last encode."""
        d = ctypes.c_uint32(0)
        r = ctypes.c_uint32(0)
        check("encoder_acsnet_stats", self._L.cujpegxl_b200_encoder_acsnet_stats(self._h, ctypes.byref(d),
                                                                                 ctypes.byref(r)))
        return d.value, r.value

    def memory(self) -> tuple[int, int]:
        """(device bytes, pinned host bytes) the encoder holds."""
        d = ctypes.c_size_t(0)
        p = ctypes.c_size_t(0)
        check("encoder_memory", self._L.cujpegxl_b200_encoder_memory(self._h, ctypes.byref(d), ctypes.byref(p)))
        return d.value, p.value


class Batch:
    """Frames of different sizes encoded by one CUDA graph launch
    (cujpegxl_b200_batch_*). `frames` lists (width, height, distance)."""

    def __init__(self, frames: list[tuple[int, int, float]], device_ordinal: int = 0):
        self._L = _capi.lib()
        self.frames = list(frames)
        cfgs = (_capi.Config * len(self.frames))(*[_capi.Config(w, h, d, device_ordinal) for w, h, d in self.frames])
        h = ctypes.c_void_p()
        check("batch_create", self._L.cujpegxl_b200_batch_create(cfgs, len(self.frames), ctypes.byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.cujpegxl_b200_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def encode(self, inputs: list[tuple[int, int, int, int]]) -> None:
        """Enqueues the batch; inputs[i] = (luma, chroma, luma_pitch, chroma_pitch) device addresses."""
        arr = (_capi.Nv12Input * len(inputs))(*[_capi.Nv12Input(*x) for x in inputs])
        check("batch_encode", self._L.cujpegxl_b200_batch_encode(self._h, arr))

    def sync(self) -> list[int]:
        sizes = (ctypes.c_size_t * len(self.frames))()
        check("batch_sync", self._L.cujpegxl_b200_batch_sync(self._h, sizes))
        return list(sizes)

    def frame(self, index: int) -> tuple[int, int]:
        """(size, device address) of a frame's file after sync."""
        size = ctypes.c_size_t(0)
        dev = ctypes.c_size_t(0)
        check("batch_frame", self._L.cujpegxl_b200_batch_frame(self._h, index, ctypes.byref(size), ctypes.byref(dev)))
        return size.value, dev.value

    def read(self, index: int) -> bytes:
        size, _ = self.frame(index)
        buf = np.empty(max(size, 1), dtype=np.uint8)
        out = _capi.Output(buf.ctypes.data, 0, buf.size)
        check("batch_copy", self._L.cujpegxl_b200_batch_copy(self._h, index, ctypes.byref(out)))
        return buf[:out.size].tobytes()

    def set_acsnet(self, net, margin: float = 0.2, flags: int = 1) -> None:
        """Learned transform decisions for every frame (see Encoder.set_acsnet);
        the next encode captures and tunes the graph again."""
        check("batch_set_acsnet", self._L.cujpegxl_b200_batch_set_acsnet(
            self._h, None if net is None else net.handle, margin, flags))
        self._net = net

    @property
    def lanes(self) -> int:
        return int(self._L.cujpegxl_b200_batch_lanes(self._h))

    def schedule(self) -> dict:
        """The frontend schedule the batch's autotuner chose (after the first
        encode): resident CTAs, tiles per claim, dynamic or round-robin
        claims, frame order, whether it came from an earlier batch of the same
        geometry mix, its measured batch time and the tiles each CTA runs at
        a time."""
        s = _capi.BatchSchedule()
        check("batch_schedule", self._L.cujpegxl_b200_batch_schedule(self._h, ctypes.byref(s)))
        return {"frontend_ctas": s.frontend_ctas, "tiles_per_claim": s.tiles_per_claim,
                "claims": "dynamic" if s.dynamic_claims else "round-robin",
                "order": "largest first" if s.largest_first else "given", "from_cache": bool(s.from_cache),
                "candidates": s.candidates, "tuned_ms": s.tuned_ms, "tiles_per_cta": s.tiles_per_cta}

    def stream(self) -> int:
        s = ctypes.c_size_t(0)
        check("batch_stream", self._L.cujpegxl_b200_batch_stream(self._h, ctypes.byref(s)))
        return s.value


def _nv12_checked(nv12: np.ndarray, width: int, height: int) -> np.ndarray:
    a = np.asarray(nv12)
    if a.dtype != np.uint8:
        raise ValueError("nv12 array must hold uint8")
    if a.size != width * height * 3 // 2:
        raise ValueError("nv12 array must hold width*height*3/2 bytes")
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("nv12 array must be C-contiguous")
    return a


def encode(nv12: np.ndarray, width: int, height: int, distance: float = 1.0, device_ordinal: int = 0) -> bytes:
    """Host NV12 -> .jxl bytes (pycujpegxl.encode)."""
    a = _nv12_checked(nv12, width, height)
    try:
        with Encoder(width, height, distance, device_ordinal) as enc:
            return enc.encode_host(a)
    except CujpegxlError as err:
        raise RuntimeError("encode failed") from err


def encode_with_stats(nv12: np.ndarray, width: int, height: int, distance: float = 1.0,
                      device_ordinal: int = 0) -> tuple[bytes, list[dict]]:
    """pycujpegxl.encode_with_stats: the bytes plus per-stage records with the
    reference's keys (name, bytes_moved, gpu_us, cpu_us)."""
    a = _nv12_checked(nv12, width, height)
    try:
        with Encoder(width, height, distance, device_ordinal) as enc:
            t0 = time.perf_counter()
            data = enc.encode_host(a)
            wall_us = (time.perf_counter() - t0) * 1e6
    except CujpegxlError as err:
        raise RuntimeError("encode failed") from err
    p = width * height
    records = [{"name": "encode", "bytes_moved": int(1.5 * p + len(data)), "gpu_us": wall_us, "cpu_us": 0.0}]
    return data, records
