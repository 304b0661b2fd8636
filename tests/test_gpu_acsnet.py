"""Transform-decision network on the GPU: the BF16 forward, loss gradient and
Adam kernels against the CPU oracle, training, and the decisions an encode
takes from the network (through the C ABI)."""

from __future__ import annotations

import numpy as np
import pytest

from cujpegxl_b200 import Encoder, acsnet
from cujpegxl_b200.decode import decode, psnr_y
from cujpegxl_b200.synth import make_nv12
from oracle import acsnet as orc

pytestmark = pytest.mark.gpu

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


def _params(seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    p = acsnet.init_params(seed)
    p[acsnet.OFF_B:acsnet.OFF_B + 3 * acsnet.C] = rng.normal(0, 0.05, 3 * acsnet.C)
    p[acsnet.OFF_B + 3 * acsnet.C:acsnet.OFF_B + 3 * acsnet.C + 1 + acsnet.NCLS] = rng.normal(0, 0.5, 18)
    return p


def _dev(tiles, l2d, labels=None, lq=None):
    import torch
    d = {"tiles": torch.from_numpy(tiles).cuda(),
         "tile_index": torch.arange(len(l2d), dtype=torch.int32).cuda(),
         "log2d": torch.from_numpy(np.asarray(l2d, np.float32)).cuda()}
    if labels is not None:
        d["label_class"] = torch.from_numpy(np.asarray(labels, np.int8)).cuda()
        d["label_qf"] = torch.from_numpy(np.asarray(lq, np.float32)).cuda()
    return d


def _rel(a, b) -> float:
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def test_forward_matches_oracle():
    """Split logits and log2 quant fields of 24 regions: relative L2 error
    against the oracle below 1e-2 (BF16 activations, FP32 accumulation)."""
    p = _params(4)
    tiles = _tiles(24, 1)
    l2d = np.linspace(-1.0, 2.0, 24)
    d = _dev(tiles, l2d)
    with acsnet.Trainer(p, NORM, 64) as tr:
        out = tr.forward(d["tiles"], d["tile_index"], d["log2d"]).cpu().numpy()
    ref = np.array([np.concatenate(orc.head(orc.forward(p, NORM, tiles[i], l2d[i])["out"])) for i in range(24)])
    assert out.shape == (24, 33)
    assert _rel(out[:, :17], ref[:, :17]) < 1e-2
    assert _rel(out[:, 17:], ref[:, 17:]) < 1e-2


def test_gradient_matches_oracle():
    """Loss gradient of a 12-sample batch, per layer and for the biases:
    relative L2 error against the oracle (same rounding points) below 3e-2."""
    rng = np.random.default_rng(8)
    p = _params(6)
    tiles = _tiles(12, 2)
    l2d = rng.uniform(-1, 2, 12)
    lab = rng.integers(0, 17, 12)
    lq = rng.uniform(1, 6, (12, 16))
    d = _dev(tiles, l2d, lab, lq)
    with acsnet.Trainer(p, NORM, 16) as tr:
        g, st = tr.gradient(d["tiles"], d["tile_index"], d["log2d"], d["label_class"], d["label_qf"], 0.7)
        g2, _ = tr.gradient(d["tiles"], d["tile_index"], d["log2d"], d["label_class"], d["label_qf"], 0.7)
        g = g.cpu().numpy()
        assert np.array_equal(g, g2.cpu().numpy()), "training must be deterministic"
        st = st.cpu().numpy()
    loss, ost, og = orc.loss_and_grad(p, NORM, tiles, l2d, lab, lq, 0.7, rnd=True)
    for layer in range(4):
        sl = slice(orc.OFF_W[layer], orc.OFF_W[layer] + orc.C * orc.KS[layer])
        assert _rel(g[sl], og[sl]) < 3e-2, f"layer {layer + 1}"
        bl = slice(orc.OFF_B + layer * orc.C, orc.OFF_B + (layer + 1) * orc.C)
        assert _rel(g[bl], og[bl]) < 3e-2, f"bias {layer + 1}"
    assert np.allclose(st[:, 0], ost[:, 0], rtol=1e-2, atol=1e-3)
    assert np.allclose(st[:, 1], ost[:, 1], rtol=1e-2, atol=1e-3)
    # Padding connections get exactly zero gradient.
    w1 = g[:orc.C * orc.K1].reshape(orc.C, orc.K1)
    assert np.all(w1[:, 72:] == 0) and np.all(w1[:, :72].reshape(orc.C, 9, 8)[:, :, 4:] == 0)


def test_soft_target_gradient_matches_oracle():
    """The same with soft split targets (a distribution over the 17 splits)."""
    import torch
    rng = np.random.default_rng(21)
    p = _params(7)
    tiles = _tiles(10, 5)
    l2d = rng.uniform(-1, 2, 10)
    lab = rng.integers(0, 17, 10)
    lq = rng.uniform(1, 6, (10, 16))
    soft = rng.dirichlet(np.full(17, 0.3), 10).astype(np.float32)
    d = _dev(tiles, l2d, lab, lq)
    with acsnet.Trainer(p, NORM, 16) as tr:
        g, st = tr.gradient(d["tiles"], d["tile_index"], d["log2d"], d["label_class"], d["label_qf"], 0.3,
                            label_soft=torch.from_numpy(soft).cuda())
        g = g.cpu().numpy()
        st = st.cpu().numpy()
    _, ost, og = orc.loss_and_grad(p, NORM, tiles, l2d, lab, lq, 0.3, rnd=True, soft=soft)
    for layer in range(4):
        sl = slice(orc.OFF_W[layer], orc.OFF_W[layer] + orc.C * orc.KS[layer])
        assert _rel(g[sl], og[sl]) < 3e-2, f"layer {layer + 1}"
    assert np.allclose(st[:, 0], ost[:, 0], rtol=1e-2, atol=1e-3)


def test_selection_costs_reproduce_the_heuristic():
    """The selection-cost planes of a debug encode give, per full region, 17
    split costs whose cheapest is the split the encode chose (ties aside)."""
    w, h = 1920, 1080
    _, planes, _ = _encode(make_nv12(w, h, 13), w, h, 1.0, debug=True)
    got = np.argmin(acsnet.class_costs(planes["cost"], w, h), axis=-1)
    want = acsnet.split_classes(planes["acs"], w, h)
    assert np.mean(got == want) > 0.995


def test_adam_step():
    """One Adam step from zero moments moves each parameter by lr * g / (|g| + eps)."""
    rng = np.random.default_rng(3)
    p = _params(9)
    tiles = _tiles(8, 4)
    d = _dev(tiles, rng.uniform(-1, 2, 8), rng.integers(0, 17, 8), rng.uniform(1, 6, (8, 16)))
    args = (d["tiles"], d["tile_index"], d["log2d"], d["label_class"], d["label_qf"], 1.0)
    with acsnet.Trainer(p, NORM, 8) as tr:
        g = tr.gradient(*args)[0].cpu().numpy().astype(np.float64)
        tr.step(*args, lr=1e-3)
        q = tr.params().astype(np.float64)
    expect = p - 1e-3 * g / (np.abs(g) + 1e-8)
    assert np.max(np.abs(q - expect)) < 1e-6


def test_training_learns_heuristic_labels():
    """A few hundred steps on one frame's labels raise the split accuracy
    well above the untrained network's."""
    data = acsnet.build_dataset([(1920, 1080, 7)], [1.0, 2.0], log=lambda *_: None)
    norm = acsnet.normalisation(data)
    with acsnet.Trainer(acsnet.init_params(1), norm, 512) as tr:
        before = acsnet.evaluate(tr, data)
    params, _, curve = acsnet.train(data, steps=400, batch=256, lr=3e-3, qf_weight=1.0, seed=1,
                                    log=lambda *_: None, norm=norm)
    with acsnet.Trainer(params, norm, 512) as tr:
        after = acsnet.evaluate(tr, data)
    assert curve[-1]["ce"] < curve[0]["ce"]
    assert after["accuracy"] > before["accuracy"] + 0.2
    assert after["qf_rmse_log2"] < before["qf_rmse_log2"]


def _net(params: np.ndarray, norm=NORM) -> acsnet.AcsNet:
    return acsnet.AcsNet(acsnet.pack_blob(params, norm))


def _encode(nv12, w, h, d, net=None, margin=0.2, flags=1, debug=False):
    with Encoder(w, h, d) as enc:
        if net is not None:
            enc.set_acsnet(net, margin, flags)
        if debug:
            enc.set_debug(True)
        data = enc.encode_host(nv12)
        planes = enc.read_planes(debug=debug)
        stats = enc.acsnet_stats() if net is not None else None
        enc.set_acsnet(None)
    return data, planes, stats


def test_unsure_network_changes_nothing():
    """A network with all-zero weights has equal logits everywhere (margin 0):
    every region falls back and the file is byte-identical to the plain path."""
    w, h = 1920, 1080
    nv12 = make_nv12(w, h, 3)
    plain, _, _ = _encode(nv12, w, h, 1.0)
    net = _net(np.zeros(acsnet.NPARAMS, np.float32))
    for flags in (acsnet.SPLIT, acsnet.SPLIT | acsnet.QF):
        got, _, stats = _encode(nv12, w, h, 1.0, net, 0.2, flags)
        assert got == plain
        assert stats == (0, (w // 32) * (h // 32))


def test_confident_network_sets_every_full_region():
    """A network biased hard towards one class decides every full region with
    it; the ragged bottom row keeps the heuristic; the file decodes."""
    w, h = 1920, 1080
    nv12 = make_nv12(w, h, 5)
    p = np.zeros(acsnet.NPARAMS, np.float32)
    cls = 6  # quadrants 0 and 2 as four DCT8, quadrants 1 and 3 as DCT16
    p[acsnet.OFF_B + 3 * acsnet.C + 1 + cls] = 40.0
    p[acsnet.OFF_B + 3 * acsnet.C] = np.log2(37.0)  # quant field 37 where QF is used
    plain, pplanes, _ = _encode(nv12, w, h, 1.0)
    data, planes, stats = _encode(nv12, w, h, 1.0, _net(p), 0.2, acsnet.SPLIT | acsnet.QF)
    assert stats == ((w // 32) * (h // 32), (w // 32) * (h // 32))
    c = acsnet.split_classes(planes["acs"], w, h)
    assert np.all(c == cls)
    bw, bh = w // 8, h // 8
    acs = planes["acs"].reshape(bh, bw)
    pacs = pplanes["acs"].reshape(bh, bw)
    assert np.array_equal(acs[4 * (h // 32):], pacs[4 * (h // 32):])
    qf = planes["qf"].reshape(bh, bw)
    assert np.all(qf[:4 * (h // 32)] == 37)
    assert np.array_equal(qf[4 * (h // 32):], pplanes["qf"].reshape(bh, bw)[4 * (h // 32):])
    img = decode(data)
    assert (img.width, img.height) == (w, h)
    assert psnr_y(nv12, data) > 35.0


def test_encoder_decisions_match_oracle():
    """Per region, the encode follows the oracle's decision on the same XYB
    tile: the network's class where the oracle margin is clearly above the
    threshold (and the oracle's quant fields within 1), the heuristic's
    split where it is clearly below."""
    w, h = 1920, 1080
    nv12 = make_nv12(w, h, 9)
    p = _params(12)
    p[acsnet.OFF_B + 3 * acsnet.C + 1:acsnet.OFF_B + 3 * acsnet.C + 18] = np.linspace(0, 1.2, 17)
    norm = np.array([40.0, 6.0, 6.0, 1.0, 0.0, 0.45, 0.45, 0.0], np.float32)
    margin = 0.1
    plain, pplanes, _ = _encode(nv12, w, h, 1.0)
    _, planes, stats = _encode(nv12, w, h, 1.0, _net(p, norm), margin, acsnet.SPLIT | acsnet.QF, debug=True)
    tiles = acsnet.region_tiles(planes["xyb"], w, h)
    got = acsnet.split_classes(planes["acs"], w, h).reshape(-1)
    heur = acsnet.split_classes(pplanes["acs"], w, h).reshape(-1)
    gq = acsnet.region_qf(planes["qf"], w, h).reshape(-1, 16)
    decided = 0
    checked = 0
    for r in range(0, tiles.shape[0], 7):
        f = orc.forward(p, norm, tiles[r], 0.0)
        logits, _ = orc.head(f["out"])
        _, top, mg, _ = orc.softmax_stats(logits)
        if abs(mg - margin) < 1e-3:
            continue
        checked += 1
        cls, q = orc.decide(f["out"], margin)
        if cls >= 0:
            decided += 1
            assert got[r] == cls
            assert np.max(np.abs(gq[r] - q)) <= 1
        else:
            assert got[r] == heur[r]
    assert checked > 200 and 0 < decided < checked
    assert 0 < stats[0] < stats[1]


def test_trained_network_against_untrained():
    """The shipped network against an untrained one of the same shape, on a
    frame outside its training set: the trained network agrees with the RD
    heuristic on most regions it is sure of and is sure of many, where the
    untrained one is neither; the learned-split encode stays within 3% of the
    heuristic's size and 0.3 dB of its PSNR-Y at distance 1."""
    w, h = 1920, 1080
    data = acsnet.build_dataset([(w, h, 424242)], [1.0], log=lambda *_: None)
    params, norm = acsnet.unpack_blob(acsnet.DEFAULT_WEIGHTS.read_bytes())
    with acsnet.Trainer(params, norm, 1024) as tr:
        trained = acsnet.evaluate(tr, data)
    with acsnet.Trainer(acsnet.init_params(1), norm, 1024) as tr:
        untrained = acsnet.evaluate(tr, data)
    assert trained["coverage"] > 0.5 and trained["covered_accuracy"] > 0.8
    assert trained["accuracy"] > untrained["accuracy"] + 0.3
    assert trained["coverage"] * trained["covered_accuracy"] > 2 * untrained["coverage"] * untrained[
        "covered_accuracy"]
    nv12 = make_nv12(w, h, 424242)
    plain, _, _ = _encode(nv12, w, h, 1.0)
    learned, _, stats = _encode(nv12, w, h, 1.0, acsnet.AcsNet.load(), 0.2, acsnet.SPLIT)
    assert stats[0] > 0
    assert len(learned) < 1.03 * len(plain)
    assert psnr_y(nv12, learned) > psnr_y(nv12, plain) - 0.3
