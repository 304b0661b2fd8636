"""Seeded synthetic NV12 frames (BT.709 full range, 8-bit 4:2:0).

The reference's real-image corpora are Git-LFS pointers or network-only, so
every benchmark and parity case uses frames from this generator instead. All
draws come from numpy's PCG64 generator seeded with `seed`.

Luma = clip(rint(gradient + coloured noise + hard edges), 0, 255), then
stripe tiles are pasted in:
  * gradient 64 + 96 * (0.6 x/W + 0.4 y/H);
  * 1/f^1.5 coloured noise: white Gaussian -> FFT -> amplitude * |f|^-1.5
    with the DC term zeroed -> inverse FFT -> scaled to sigma = 12;
  * 40 hard edges: 20 axis-aligned and 20 diagonal half-plane steps, each
    confined to a random rectangle of 64..512 px per side and adding
    +-U(30, 80);
  * 8 tiles of 64x64 with 1- or 2-px-period stripes alternating 16/235,
    horizontal or vertical.
Chroma, per plane at (W/2) x (H/2): Gaussian-blurred (sigma = 8 px) white
noise normalised to +-20 peak around 128, clipped to [0, 255], interleaved
Cb/Cr with a row pitch of W bytes.
"""

from __future__ import annotations

import numpy as np


def _coloured_noise(rng: np.random.Generator, h: int, w: int, sigma: float) -> np.ndarray:
    white = rng.standard_normal((h, w))
    spec = np.fft.rfft2(white)
    fy = np.fft.fftfreq(h)[:, None]
    fx = np.fft.rfftfreq(w)[None, :]
    f = np.sqrt(fx * fx + fy * fy)
    f[0, 0] = 1.0
    amp = f ** -1.5
    amp[0, 0] = 0.0
    noise = np.fft.irfft2(spec * amp, s=(h, w))
    std = noise.std()
    return noise * (sigma / std) if std > 0 else noise


def _gaussian_blur(img: np.ndarray, sigma: float) -> np.ndarray:
    h, w = img.shape
    fy = np.fft.fftfreq(h)[:, None]
    fx = np.fft.rfftfreq(w)[None, :]
    g = np.exp(-2.0 * (np.pi * sigma) ** 2 * (fx * fx + fy * fy))
    return np.fft.irfft2(np.fft.rfft2(img) * g, s=(h, w))


def make_nv12(width: int, height: int, seed: int = 0) -> np.ndarray:
    """Returns one NV12 frame as a flat uint8 array of width*height*3/2 bytes."""
    if width % 2 or height % 2:
        raise ValueError("NV12 needs even dimensions")
    rng = np.random.Generator(np.random.PCG64(seed))
    yy, xx = np.mgrid[0:height, 0:width].astype(np.float64)
    luma = 64.0 + 96.0 * (0.6 * xx / width + 0.4 * yy / height)
    luma += _coloured_noise(rng, height, width, 12.0)

    for i in range(40):
        rw = int(rng.integers(64, 513))
        rh = int(rng.integers(64, 513))
        x0 = int(rng.integers(0, max(1, width - rw + 1)))
        y0 = int(rng.integers(0, max(1, height - rh + 1)))
        amp = float(rng.uniform(30.0, 80.0)) * (1.0 if rng.random() < 0.5 else -1.0)
        sub_y, sub_x = np.mgrid[0:min(rh, height - y0), 0:min(rw, width - x0)]
        if i < 20:
            if rng.random() < 0.5:
                mask = sub_x >= int(rng.integers(0, sub_x.shape[1]))
            else:
                mask = sub_y >= int(rng.integers(0, sub_y.shape[0]))
        else:
            angle = float(rng.uniform(0.0, np.pi))
            cx = float(rng.uniform(0, sub_x.shape[1]))
            cy = float(rng.uniform(0, sub_y.shape[0]))
            mask = (sub_x - cx) * np.cos(angle) + (sub_y - cy) * np.sin(angle) >= 0.0
        luma[y0:y0 + mask.shape[0], x0:x0 + mask.shape[1]] += amp * mask

    luma = np.clip(np.rint(luma), 0, 255)
    for _ in range(8):
        x0 = int(rng.integers(0, max(1, width - 64 + 1)))
        y0 = int(rng.integers(0, max(1, height - 64 + 1)))
        period = int(rng.integers(1, 3))
        sub_y, sub_x = np.mgrid[0:min(64, height - y0), 0:min(64, width - x0)]
        coord = sub_x if rng.random() < 0.5 else sub_y
        luma[y0:y0 + coord.shape[0], x0:x0 + coord.shape[1]] = np.where((coord // period) % 2 == 0, 16, 235)

    cw, ch = width // 2, height // 2
    planes = []
    for _ in range(2):
        p = _gaussian_blur(rng.standard_normal((ch, cw)), 8.0)
        peak = np.abs(p).max()
        p = 128.0 + (20.0 * p / peak if peak > 0 else p)
        planes.append(np.clip(np.rint(p), 0, 255))
    chroma = np.empty((ch, width), dtype=np.uint8)
    chroma[:, 0::2] = planes[0]
    chroma[:, 1::2] = planes[1]
    return np.concatenate([luma.astype(np.uint8).ravel(), chroma.ravel()])
