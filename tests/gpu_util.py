"""Helpers for the GPU tests: device NV12 frames through torch (plumbing only)."""

from __future__ import annotations

import numpy as np


def device_nv12(nv12: np.ndarray, width: int, height: int, luma_pitch: int | None = None,
                chroma_pitch: int | None = None):
    """Uploads an NV12 frame into device buffers with the given row pitches.
    Returns (keepalive, luma_address, chroma_address, luma_pitch, chroma_pitch)."""
    import torch

    lp = luma_pitch or width
    cp = chroma_pitch or width
    flat = np.ascontiguousarray(nv12, np.uint8).ravel()
    luma = np.zeros((height, lp), np.uint8)
    luma[:, :width] = flat[: width * height].reshape(height, width)
    chroma = np.zeros((height // 2, cp), np.uint8)
    chroma[:, :width] = flat[width * height:].reshape(height // 2, width)
    tl = torch.from_numpy(luma).cuda()
    tc = torch.from_numpy(chroma).cuda()
    torch.cuda.synchronize()
    return (tl, tc), tl.data_ptr(), tc.data_ptr(), lp, cp
