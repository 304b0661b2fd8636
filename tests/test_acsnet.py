"""Transform-decision network, host side (no GPU): the weights blob and its
library check, label extraction from AC-strategy planes, and the CPU oracle
pinned against finite differences."""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from cujpegxl_b200 import acsnet
from oracle import acsnet as orc

NORM = np.array([30.0, 4.0, 4.0, 1.0, 0.0, 0.4, 0.4, 0.5], np.float32)


def _tiles(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    out = np.empty((n, 3, 34, 34), np.float32)
    yy, xx = np.mgrid[0:34, 0:34] / 32.0
    for i in range(n):
        tex = rng.normal(0, rng.uniform(0.002, 0.05), (34, 34))
        out[i, 0] = rng.normal(0, 0.01) + 0.2 * tex * rng.uniform(0, 1)
        out[i, 1] = 0.4 + 0.2 * (xx * rng.uniform(-1, 1) + yy * rng.uniform(-1, 1)) + tex
        out[i, 2] = out[i, 1] + rng.normal(0, 0.02)
    return out


def test_library_constants_match_python():
    assert acsnet.NPARAMS == orc.NPARAMS == 30336
    from cujpegxl_b200 import _capi
    assert _capi.lib().cujpegxl_b200_acsnet_param_count() == acsnet.NPARAMS


def test_blob_round_trip_and_library_check():
    p = acsnet.init_params(7)
    blob = acsnet.pack_blob(p, NORM)
    assert len(blob) == 4 + 24 + 32 + 4 * acsnet.NPARAMS + 32
    assert hashlib.sha256(blob[:-32]).digest() == blob[-32:]
    assert acsnet.check_blob(blob)
    q, n = acsnet.unpack_blob(blob)
    assert np.array_equal(q, p) and np.array_equal(n, NORM)
    for cut in (0, 1, len(blob) - 1):
        assert not acsnet.check_blob(blob[:cut])
    for at in (0, 5, 30, 1000, len(blob) - 40, len(blob) - 1):
        bad = bytearray(blob)
        bad[at] ^= 0x10
        assert not acsnet.check_blob(bytes(bad))
        with pytest.raises(ValueError):
            acsnet.unpack_blob(bytes(bad))
    # A non-finite parameter is refused even with a matching checksum.
    p2 = p.copy()
    p2[123] = np.inf
    assert not acsnet.check_blob(acsnet.pack_blob(p2, NORM))


def test_shipped_weights_blob():
    blob = acsnet.DEFAULT_WEIGHTS.read_bytes()
    assert acsnet.check_blob(blob)
    params, norm = acsnet.unpack_blob(blob)
    assert np.all(np.isfinite(params)) and np.all(norm[:4] > 0)
    # Connections that must stay zero (unused input channels, L1 padding
    # columns, unused L4 output channels) are zero.
    w1 = params[:acsnet.C * acsnet.K1].reshape(acsnet.C, acsnet.K1)
    assert np.all(w1[:, 72:] == 0)
    assert np.all(w1[:, :72].reshape(acsnet.C, 9, 8)[:, :, 4:] == 0)
    w4 = params[acsnet.OFF_W[3]:acsnet.OFF_W[3] + acsnet.C * acsnet.K].reshape(acsnet.C, acsnet.K)
    assert np.all(w4[1 + acsnet.NCLS:] == 0)


def _random_acs(rng, bw: int, bh: int) -> np.ndarray:
    acs = np.zeros((bh, bw), np.int8)
    for ry in range(bh // 4):
        for rx in range(bw // 4):
            c = int(rng.integers(0, 17))
            for dy in range(4):
                for dx in range(4):
                    q = (dy >> 1) * 2 + (dx >> 1)
                    if c == 0:
                        v = 32 if dx == 0 and dy == 0 else 0
                    elif ((c - 1) >> q) & 1:
                        v = 8
                    else:
                        v = 16 if (dx & 1) == 0 and (dy & 1) == 0 else 0
                    acs[4 * ry + dy, 4 * rx + dx] = v
    # Ragged edge blocks (not a full region) use DCT8.
    acs[4 * (bh // 4):, :] = 8
    acs[:, 4 * (bw // 4):] = 8
    return acs


@pytest.mark.parametrize("w,h", [(128, 96), (200, 136)])
def test_split_classes_match_oracle(w, h):
    rng = np.random.default_rng(w + h)
    bw, bh = w // 8, h // 8
    acs = _random_acs(rng, bw, bh)
    got = acsnet.split_classes(acs.reshape(-1), w, h)
    assert got.shape == (h // 32, w // 32)
    for ry in range(h // 32):
        for rx in range(w // 32):
            assert got[ry, rx] == orc.split_class(acs[4 * ry:4 * ry + 4, 4 * rx:4 * rx + 4])
    qf = rng.integers(1, 257, (bh, bw)).astype(np.int32)
    rq = acsnet.region_qf(qf.reshape(-1), w, h)
    assert np.array_equal(rq[1, 0], qf[4:8, 0:4].reshape(16))
    xyb = rng.normal(size=(3, h, w)).astype(np.float32)
    t = acsnet.region_tiles(xyb, w, h)
    assert t.shape == ((h // 32) * (w // 32), 3, 34, 34)
    assert np.array_equal(t[(w // 32) + 1], xyb[:, 31:65, 31:65])
    # The ring is clamped to the image at its border.
    assert np.array_equal(t[0][:, 1:, 1:], xyb[:, :33, :33])
    assert np.array_equal(t[0][:, 0, 1:], xyb[:, 0, :33]) and np.array_equal(t[0][:, 1:, 0], xyb[:, :33, 0])


def test_class_costs_argmin_is_the_rd_rule():
    """The cheapest of the 17 split costs is the split the RD rule picks
    (DCT16 over four DCT8 when not dearer, then DCT32 over the split)."""
    w, h = 256, 192
    bw, bh = w // 8, h // 8
    rng = np.random.default_rng(4)
    cost = np.zeros((3, bh, bw), np.float32)
    cost[0] = rng.uniform(10, 20, (bh, bw))
    cost[1][0::2, 0::2] = rng.uniform(25, 95, (bh // 2, bw // 2))
    cost[2][0::4, 0::4] = rng.uniform(100, 330, (bh // 4, bw // 4))
    cc = acsnet.class_costs(cost.reshape(-1), w, h)
    for ry in range(h // 32):
        for rx in range(w // 32):
            split, m = 0.0, 0
            for q in range(4):
                by, bx = 4 * ry + 2 * (q >> 1), 4 * rx + 2 * (q & 1)
                s8 = float(cost[0][by:by + 2, bx:bx + 2].sum())
                c16 = float(cost[1][by, bx])
                if c16 <= s8:
                    split += c16
                else:
                    split += s8
                    m |= 1 << q
            want = 0 if cost[2][4 * ry, 4 * rx] <= split else 1 + m
            assert int(np.argmin(cc[ry, rx])) == want
            assert np.isclose(cc[ry, rx].min(), min(split, cost[2][4 * ry, 4 * rx]))


def test_oracle_gradient_matches_finite_differences():
    """Pins the oracle: its analytic gradient (rounding off) against central
    differences of its own loss, relative L2 error below 1e-3."""
    rng = np.random.default_rng(5)
    p = acsnet.init_params(11).astype(np.float64)
    p[orc.OFF_B:] = rng.normal(0, 0.05, 4 * orc.C)
    p[orc.OFF_B + 3 * orc.C + 1 + orc.NCLS:] = 0.0
    tiles = _tiles(2, 3)
    l2d = np.array([0.0, 1.0])
    lab = np.array([5, 0])
    lq = rng.uniform(1, 5, (2, 16))
    _, _, g = orc.loss_and_grad(p, NORM, tiles, l2d, lab, lq, 0.5, rnd=False)
    live = np.nonzero(g)[0]
    idx = np.concatenate([rng.choice(live[live < orc.NW], 40, replace=False),
                          rng.choice(live[live >= orc.NW], 8, replace=False)])
    fd = []
    for i in idx:
        q = p.copy()
        q[i] += 1e-5
        lp = orc.loss_and_grad(q, NORM, tiles, l2d, lab, lq, 0.5, rnd=False)[0]
        q[i] -= 2e-5
        lm = orc.loss_and_grad(q, NORM, tiles, l2d, lab, lq, 0.5, rnd=False)[0]
        fd.append((lp - lm) / 2e-5)
    fd = np.array(fd)
    assert np.linalg.norm(fd - g[idx]) / np.linalg.norm(g[idx]) < 1e-3


def test_oracle_rounding_is_small():
    """BF16 rounding at the kernel's rounding points moves the loss gradient
    by a few percent at most (relative L2)."""
    p = acsnet.init_params(2)
    tiles = _tiles(3, 9)
    args = (NORM, tiles, np.array([0.0, 1.0, -1.0]), np.array([1, 16, 0]), np.full((3, 16), 3.0), 1.0)
    _, _, g0 = orc.loss_and_grad(p, *args, rnd=False)
    _, _, g1 = orc.loss_and_grad(p, *args, rnd=True)
    assert np.linalg.norm(g1 - g0) / np.linalg.norm(g0) < 0.05
