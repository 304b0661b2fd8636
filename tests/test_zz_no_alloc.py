"""cujpegxl_b200_encode_planes_noalloc: the allocation-free entry point for
callers that cannot allocate device memory while they encode (a real-time
loop where cudaMalloc would synchronise the device, or device memory held
entirely by the caller's own pool).

Through the C ABI it must produce exactly the file that the allocating entry
point cujpegxl_b200_encode_planes produces for the same planes, on two calls
in a row (the second call reuses the shared scratch array left by the first),
and reject frames above its 4-megapixel limit. This file is collected last so
that a run stopping at the first failure has run every other test already.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from cujpegxl_b200 import Encoder, _capi

from . import patterns as P

pytestmark = pytest.mark.gpu


def _device_planes(f: dict):
    import torch

    flat = P.flat(f)
    keep = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in flat.items()}
    torch.cuda.synchronize()
    dp = _capi.DevicePlanes(*[keep[k].data_ptr() for k in ("ac", "dc", "acs", "qf", "ytox", "ytob")])
    return keep, dp


def _device_planes_flat(planes: dict):
    import torch

    keep = {k: torch.from_numpy(np.ascontiguousarray(planes[k])).cuda()
            for k in ("ac", "dc", "acs", "qf", "ytox", "ytob")}
    torch.cuda.synchronize()
    dp = _capi.DevicePlanes(*[keep[k].data_ptr() for k in ("ac", "dc", "acs", "qf", "ytox", "ytob")])
    return keep, dp


def _noalloc(dp, w: int, h: int, gs: int, qdc: int, out, capacity: int) -> tuple[int, int]:
    size = ctypes.c_size_t(0)
    code = _capi.lib().cujpegxl_b200_encode_planes_noalloc(ctypes.byref(dp), w, h, gs, qdc, out.data_ptr(),
                                                          capacity, ctypes.byref(size), 0)
    return code, size.value


@pytest.mark.parametrize("w,h,seed", [(512, 384, None), (1024, 768, 7)])
def test_noalloc_matches_allocating_entry_point_twice(w, h, seed):
    import torch

    f = P.mixed_full(w, h, seed=seed)
    if seed is None:
        P.fill_ac_pattern(f)
    gs, qdc = 4096, 32
    with Encoder(w, h, 1.0) as enc:
        expected = enc.encode_planes(P.flat(f), gs, qdc)
    keep, dp = _device_planes(f)
    cap = 4 << 20
    out = torch.empty(cap, dtype=torch.uint8, device="cuda")
    for _ in range(2):
        out.fill_(0xA5)
        code, size = _noalloc(dp, w, h, gs, qdc, out, cap)
        assert code == _capi.OK, _capi.status_string(code)
        assert size == len(expected)
        assert out[:size].cpu().numpy().tobytes() == expected


@pytest.mark.parametrize("w,h", [(2048, 2048), (4096, 1024)])
def test_noalloc_real_planes_at_limit_and_multi_dc_group(w, h):
    """Planes of a real encode at the 4-megapixel limit (2048x2048: 64 AC
    groups, 4 DC groups) and of a wide frame (4096x1024: 2 DC-group rows of
    two): the file equals the allocating encoder's own, twice in a row."""
    import torch

    from cujpegxl_b200.synth import make_nv12
    from oracle import api

    from .gpu_util import device_nv12

    nv12 = make_nv12(w, h, 3)
    keep_in, lum, chrom, lp, cp = device_nv12(nv12, w, h)
    with Encoder(w, h, 1.0) as enc:
        expected = enc.encode_device(lum, chrom, lp, cp)
        planes = enc.read_planes()
    sc = api.scalars(1.0)
    keep, dp = _device_planes_flat(planes)
    cap = 8 << 20
    out = torch.empty(cap, dtype=torch.uint8, device="cuda")
    for _ in range(2):
        out.fill_(0x5A)
        code, size = _noalloc(dp, w, h, sc["global_scale"], sc["quant_dc"], out, cap)
        assert code == _capi.OK, _capi.status_string(code)
        assert size == len(expected)
        assert out[:size].cpu().numpy().tobytes() == expected


def test_noalloc_rejects_misaligned_planes():
    import torch

    keep, dp = _device_planes(P.mixed_full(512, 384))
    out = torch.empty(1 << 20, dtype=torch.uint8, device="cuda")
    for field in ("dc", "qf", "ac"):
        bad = _capi.DevicePlanes(*[getattr(dp, k) + (2 if k == field else 0)
                                   for k in ("ac", "dc", "acs", "qf", "ytox", "ytob")])
        code, _ = _noalloc(bad, 512, 384, 4096, 32, out, out.numel())
        assert code == _capi.INVALID_ARGUMENT, field


def test_noalloc_rejects_frames_above_limit_and_small_buffers():
    import torch

    keep, dp = _device_planes(P.mixed_full(512, 384))
    out = torch.empty(1 << 20, dtype=torch.uint8, device="cuda")
    code, _ = _noalloc(dp, 2560, 2304, 4096, 32, out, out.numel())    # 5.9 MP > 4 MP
    assert code == _capi.UNSUPPORTED_RESOLUTION
    code, size = _noalloc(dp, 512, 384, 4096, 32, out, 64)
    assert code == _capi.BUFFER_TOO_SMALL and size > 64
