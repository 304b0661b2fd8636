"""Learned transform decisions: weights blobs, the network handle, and the GPU
training pipeline.

The network (csrc/acsnet.cuh) looks at one 32x32 region of XYB pixels and the
distance, and predicts the region's DCT32/DCT16/DCT8 split and the quant field
of its 16 blocks. It is trained on labels the plain RD heuristic and adaptive
quantisation produce on seeded synthetic frames, entirely on the GPU by the
library's own BF16 kernels (forward, backward, Adam); at encode time regions
where its softmax margin is below a threshold keep the heuristic.

    python -m cujpegxl_b200.acsnet --out cujpegxl_b200/data/acsnet_v2.jxbn

trains the shipped weights (about a minute on one B200) and writes a JSON
report beside them.
"""

from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import math
import struct
import time
from pathlib import Path

import numpy as np

from . import _capi
from ._capi import check

C = 32
NCLS = 17
K1 = 80
K = 288
OFF_W = (0, C * K1, C * K1 + C * K, C * K1 + 2 * C * K)
NW = C * K1 + 3 * C * K
OFF_B = NW
NPARAMS = NW + 4 * C
MAGIC = b"JXBN"
VERSION = 2
SPLIT = 1
QF = 2
DEFAULT_MARGIN = 0.2
DEFAULT_WEIGHTS = Path(__file__).resolve().parent / "data" / "acsnet_v2.jxbn"


def pack_blob(params: np.ndarray, norm: np.ndarray) -> bytes:
    """Weights blob: header, scale[4], shift[4], FP32 parameters, SHA-256."""
    p = np.ascontiguousarray(params, np.float32).reshape(-1)
    n = np.ascontiguousarray(norm, np.float32).reshape(-1)
    if p.size != NPARAMS or n.size != 8:
        raise ValueError("parameter or normalisation size")
    body = MAGIC + struct.pack("<6I", VERSION, NPARAMS, C, NCLS, K1, K) + n.astype("<f4").tobytes() + \
        p.astype("<f4").tobytes()
    return body + hashlib.sha256(body).digest()


def unpack_blob(blob: bytes) -> tuple[np.ndarray, np.ndarray]:
    """(parameters, normalisation) of a blob; ValueError if it is malformed."""
    if len(blob) != 4 + 24 + 32 + 4 * NPARAMS + 32 or blob[:4] != MAGIC:
        raise ValueError("not a transform-decision network blob")
    if struct.unpack("<6I", blob[4:28]) != (VERSION, NPARAMS, C, NCLS, K1, K):
        raise ValueError("unsupported network version or geometry")
    if hashlib.sha256(blob[:-32]).digest() != blob[-32:]:
        raise ValueError("blob checksum mismatch")
    norm = np.frombuffer(blob[28:60], "<f4").astype(np.float32)
    params = np.frombuffer(blob[60:-32], "<f4").astype(np.float32)
    return params, norm


def init_params(seed: int) -> np.ndarray:
    """He-normal weights on the live connections (X, Y, B and log2 distance
    into L1; channels 0..17 out of L4), zeros elsewhere and for the biases."""
    rng = np.random.Generator(np.random.PCG64(seed))
    p = np.zeros(NPARAMS, np.float32)
    w1 = np.zeros((C, 9, 8), np.float32)
    w1[:, :, :4] = rng.standard_normal((C, 9, 4)) * math.sqrt(2.0 / 36.0)
    full = np.zeros((C, K1), np.float32)
    full[:, :72] = w1.reshape(C, 72)
    p[OFF_W[0]:OFF_W[0] + C * K1] = full.reshape(-1)
    for layer in (1, 2):
        p[OFF_W[layer]:OFF_W[layer] + C * K] = (rng.standard_normal((C, K)) * math.sqrt(2.0 / K)).reshape(-1)
    w4 = np.zeros((C, K), np.float32)
    w4[:1 + NCLS] = rng.standard_normal((1 + NCLS, K)) * math.sqrt(1.0 / K)
    p[OFF_W[3]:OFF_W[3] + C * K] = w4.reshape(-1)
    return p


def split_classes(acs: np.ndarray, width: int, height: int) -> np.ndarray:
    """Split class of every full 32x32 region ([H/32][W/32], int8) from a
    block-raster AC-strategy plane (side at first blocks, 0 elsewhere):
    0 = DCT32, 1 + m = quadrant q four DCT8 when bit q of m is set, else DCT16;
    -1 where the region is not such a split."""
    bw, bh = width // 8, height // 8
    rw, rh = width // 32, height // 32
    a = np.asarray(acs, np.int8).reshape(bh, bw)[:4 * rh, :4 * rw].reshape(rh, 4, rw, 4).transpose(0, 2, 1, 3)
    tops = np.stack([a[:, :, 2 * (q >> 1), 2 * (q & 1)] for q in range(4)], axis=-1)
    m = ((tops == 8).astype(np.int32) << np.arange(4)).sum(axis=-1)
    ok_split = np.all((tops == 8) | (tops == 16), axis=-1)
    return np.where(a[:, :, 0, 0] == 32, 0, np.where(ok_split, 1 + m, -1)).astype(np.int8)


def region_qf(qf: np.ndarray, width: int, height: int) -> np.ndarray:
    """Quant field of the blocks of every full region, [H/32][W/32][16]."""
    bw, bh = width // 8, height // 8
    rw, rh = width // 32, height // 32
    q = np.asarray(qf).reshape(bh, bw)[:4 * rh, :4 * rw].reshape(rh, 4, rw, 4).transpose(0, 2, 1, 3)
    return q.reshape(rh, rw, 16)


def region_tiles(xyb: np.ndarray, width: int, height: int) -> np.ndarray:
    """[H/32 * W/32][3][34][34] XYB inputs of the full regions, raster order:
    each region with a 1-pixel ring of its neighbours (coordinates clamped to
    the image, as the inference kernel reads them)."""
    rw, rh = width // 32, height // 32
    x = np.pad(np.asarray(xyb, np.float32).reshape(3, height, width), ((0, 0), (1, 1), (1, 1)), mode="edge")
    out = np.empty((rh * rw, 3, 34, 34), np.float32)
    for ry in range(rh):
        for rx in range(rw):
            out[ry * rw + rx] = x[:, 32 * ry:32 * ry + 34, 32 * rx:32 * rx + 34]
    return out


def class_costs(cost: np.ndarray, width: int, height: int) -> np.ndarray:
    """RD cost of each of the 17 splits of every full region, [H/32][W/32][17],
    from the selection-cost planes ([3][B]: DCT8 per block, DCT16 at quad and
    DCT32 at region first blocks). Their arg-min is the heuristic's choice."""
    bw, bh = width // 8, height // 8
    rw, rh = width // 32, height // 32
    c = np.asarray(cost, np.float64).reshape(3, bh, bw)[:, :4 * rh, :4 * rw]
    c = c.reshape(3, rh, 4, rw, 4).transpose(0, 1, 3, 2, 4)  # [3][rh][rw][4][4]
    c8 = c[0].reshape(rh, rw, 2, 2, 2, 2).sum(axis=(3, 5)).reshape(rh, rw, 4)
    c16 = c[1][:, :, 0::2, 0::2].reshape(rh, rw, 4)
    out = np.empty((rh, rw, NCLS), np.float64)
    out[..., 0] = c[2][:, :, 0, 0]
    for m in range(16):
        bits = np.array([(m >> q) & 1 for q in range(4)], bool)
        out[..., 1 + m] = np.where(bits, c8, c16).sum(axis=-1)
    return out


class AcsNet:
    """A transform-decision network uploaded to one device."""

    def __init__(self, blob: bytes, device_ordinal: int = 0):
        self._L = _capi.lib()
        self._h = ctypes.c_void_p()
        buf = ctypes.create_string_buffer(bytes(blob), len(blob))
        check("acsnet_create", self._L.cujpegxl_b200_acsnet_create(buf, len(blob), device_ordinal,
                                                                   ctypes.byref(self._h)))
        self.device_ordinal = device_ordinal

    @classmethod
    def load(cls, path: str | Path = DEFAULT_WEIGHTS, device_ordinal: int = 0) -> "AcsNet":
        return cls(Path(path).read_bytes(), device_ordinal)

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def close(self) -> None:
        if self._h:
            self._L.cujpegxl_b200_acsnet_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def check_blob(blob: bytes) -> bool:
    """The library's own blob check (layout and SHA-256), no device needed."""
    buf = ctypes.create_string_buffer(bytes(blob), len(blob))
    return _capi.lib().cujpegxl_b200_acsnet_check_blob(buf, len(blob)) == _capi.OK


def _batch(tiles, tile_index, log2d, label_class=None, label_qf=None, label_soft=None) -> _capi.NetBatch:
    def p(t):
        return 0 if t is None else t.data_ptr()
    return _capi.NetBatch(p(tiles), p(tile_index), p(log2d), p(label_class), p(label_qf), int(tile_index.numel()),
                          p(label_soft))


def soft_targets(regret, temperature: float):
    """Target distribution over the 17 splits from their relative RD regret
    (cost / min cost - 1): softmax(-regret / temperature)."""
    import torch
    return torch.softmax(-regret / temperature, dim=1).float().contiguous()


class Trainer:
    """FP32 master weights, Adam state and activation scratch on the device.
    Batches are torch CUDA tensors: tiles float32 [T][3][34][34], tile_index
    int32 [n], log2d float32 [n], label_class int8 [n], label_qf float32 [n][16],
    optional label_soft float32 [n][17]."""

    def __init__(self, params: np.ndarray, norm: np.ndarray, max_batch: int, device_ordinal: int = 0):
        import torch
        self._torch = torch
        self._L = _capi.lib()
        self._h = ctypes.c_void_p()
        p = np.ascontiguousarray(params, np.float32)
        n = np.ascontiguousarray(norm, np.float32)
        check("acsnet_trainer_create", self._L.cujpegxl_b200_acsnet_trainer_create(
            p.ctypes.data, n.ctypes.data, max_batch, device_ordinal, ctypes.byref(self._h)))
        self.norm = n.copy()
        self.max_batch = max_batch
        self.device = torch.device("cuda", device_ordinal)

    def _stream(self) -> int:
        return self._torch.cuda.current_stream(self.device).cuda_stream

    def forward(self, tiles, tile_index, log2d):
        out = self._torch.empty((tile_index.numel(), NCLS + 16), dtype=self._torch.float32, device=self.device)
        b = _batch(tiles, tile_index, log2d)
        check("acsnet_trainer_forward", self._L.cujpegxl_b200_acsnet_trainer_forward(
            self._h, ctypes.byref(b), out.data_ptr(), self._stream()))
        return out

    def gradient(self, tiles, tile_index, log2d, label_class, label_qf, qf_weight: float, label_soft=None):
        t = self._torch
        grad = t.empty(NPARAMS, dtype=t.float32, device=self.device)
        stats = t.empty((tile_index.numel(), 4), dtype=t.float32, device=self.device)
        b = _batch(tiles, tile_index, log2d, label_class, label_qf, label_soft)
        check("acsnet_trainer_gradient", self._L.cujpegxl_b200_acsnet_trainer_gradient(
            self._h, ctypes.byref(b), qf_weight, grad.data_ptr(), stats.data_ptr(), self._stream()))
        return grad, stats

    def step(self, tiles, tile_index, log2d, label_class, label_qf, qf_weight: float, lr: float, stats=None,
             label_soft=None):
        b = _batch(tiles, tile_index, log2d, label_class, label_qf, label_soft)
        check("acsnet_trainer_step", self._L.cujpegxl_b200_acsnet_trainer_step(
            self._h, ctypes.byref(b), qf_weight, lr, 0 if stats is None else stats.data_ptr(), self._stream()))

    def params(self) -> np.ndarray:
        out = np.empty(NPARAMS, np.float32)
        check("acsnet_trainer_params", self._L.cujpegxl_b200_acsnet_trainer_params(self._h, out.ctypes.data))
        return out

    def close(self) -> None:
        if self._h:
            self._L.cujpegxl_b200_acsnet_trainer_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def build_dataset(frames: list[tuple[int, int, int]], distances: list[float], device_ordinal: int = 0,
                  log=print) -> dict:
    """Tiles and labels from the plain encoder on seeded synthetic frames.

    frames: (width, height, seed). Every full 32x32 region of every frame is
    one tile; each tile gets one sample per distance, labelled with the split
    the RD heuristic chose, the relative RD regret of all 17 splits
    (cost / min cost - 1) and the adaptive quant field (log2) of its blocks."""
    import torch
    from . import Encoder
    from .synth import make_nv12
    dev = torch.device("cuda", device_ordinal)
    tiles, t_idx, l2d, cls, lqf, reg = [], [], [], [], [], []
    base = 0
    for (w, h, seed) in frames:
        nv12 = make_nv12(w, h, seed)
        with Encoder(w, h, distances[0], device_ordinal) as enc:
            enc.set_debug(True)
            for d in distances:
                enc.configure(w, h, d)
                enc.encode_host(nv12)
                pl = enc.read_planes(debug=True, keys=("acs", "qf", "cost", "xyb") if d == distances[0] else
                                     ("acs", "qf", "cost"))
                if d == distances[0]:
                    tl = region_tiles(pl["xyb"], w, h)
                    tiles.append(torch.from_numpy(tl).to(dev))
                c = split_classes(pl["acs"], w, h).reshape(-1)
                q = region_qf(pl["qf"], w, h).reshape(-1, 16)
                cc = class_costs(pl["cost"], w, h).reshape(-1, NCLS)
                ok = np.nonzero(c >= 0)[0]
                t_idx.append(base + ok.astype(np.int32))
                l2d.append(np.full(ok.size, math.log2(d), np.float32))
                cls.append(c[ok])
                lqf.append(np.log2(q[ok].astype(np.float64)).astype(np.float32))
                low = cc[ok].min(axis=1, keepdims=True)
                reg.append((cc[ok] / np.maximum(low, 1e-9) - 1.0).astype(np.float32))
        base += tl.shape[0]
        log(f"dataset: {w}x{h} seed {seed}: {tl.shape[0]} tiles")
    return {
        "tiles": torch.cat(tiles),
        "tile_index": torch.from_numpy(np.concatenate(t_idx)).to(dev),
        "log2d": torch.from_numpy(np.concatenate(l2d)).to(dev),
        "label_class": torch.from_numpy(np.concatenate(cls)).to(dev),
        "label_qf": torch.from_numpy(np.concatenate(lqf)).to(dev),
        "regret": torch.from_numpy(np.concatenate(reg)).to(dev),
    }


def normalisation(data: dict) -> np.ndarray:
    """scale[4], shift[4]: zero mean and unit deviation of X, Y, B (over a
    sample of tiles) and of log2 distance."""
    t = data["tiles"]
    step = max(1, t.shape[0] // 4096)
    sub = t[::step].transpose(0, 1).reshape(3, -1).double()
    mean = sub.mean(dim=1).cpu().numpy()
    std = sub.std(dim=1).cpu().numpy()
    l2 = data["log2d"].double()
    lm, ls = float(l2.mean()), float(l2.std()) or 1.0
    scale = np.array([1.0 / max(s, 1e-6) for s in std] + [1.0 / ls], np.float32)
    shift = np.array(list(mean) + [lm], np.float32)
    return np.concatenate([scale, shift])


def evaluate(trainer: Trainer, data: dict, margin: float = DEFAULT_MARGIN) -> dict:
    """Split accuracy over all samples, the fraction with a softmax margin of
    at least `margin` and the accuracy on those, the mean relative RD regret
    of the network's split where it is sure (and over all samples, counting
    the heuristic's fallback as no regret), and the log2 quant-field RMSE."""
    import torch
    n = data["tile_index"].numel()
    correct = covered = covered_ok = 0
    sq = regret = 0.0
    for s in range(0, n, trainer.max_batch):
        e = min(n, s + trainer.max_batch)
        out = trainer.forward(data["tiles"], data["tile_index"][s:e], data["log2d"][s:e])
        prob = torch.softmax(out[:, :NCLS].double(), dim=1)
        top2 = torch.topk(prob, 2, dim=1)
        pred = top2.indices[:, 0]
        lab = data["label_class"][s:e].long()
        conf = (top2.values[:, 0] - top2.values[:, 1]) >= margin
        ok = pred == lab
        correct += int(ok.sum())
        covered += int(conf.sum())
        covered_ok += int((ok & conf).sum())
        sq += float(((out[:, NCLS:].double() - data["label_qf"][s:e].double()) ** 2).sum())
        r = data["regret"][s:e].double().gather(1, pred[:, None])[:, 0]
        regret += float((r * conf).sum())
    return {"samples": n, "accuracy": correct / n, "coverage": covered / n,
            "covered_accuracy": covered_ok / max(1, covered), "regret_covered": regret / max(1, covered),
            "regret_effective": regret / n, "qf_rmse_log2": math.sqrt(sq / (16 * n))}


def train(data: dict, *, steps: int, batch: int, lr: float, qf_weight: float, seed: int,
          device_ordinal: int = 0, log=print, params: np.ndarray | None = None,
          norm: np.ndarray | None = None, temperature: float = 0.0) -> tuple[np.ndarray, np.ndarray, list]:
    """Adam with a cosine learning-rate decay over `steps` batches drawn with
    replacement (seeded). temperature > 0 trains the split against
    soft_targets(regret, temperature) instead of the heuristic's one-hot
    choice, so that near-ties cost little and expensive mistakes much.
    Returns (params, norm, loss curve)."""
    import torch
    norm = normalisation(data) if norm is None else norm
    params = init_params(seed) if params is None else params
    n = data["tile_index"].numel()
    gen = torch.Generator(device=data["tile_index"].device)
    gen.manual_seed(seed)
    curve = []
    with Trainer(params, norm, batch, device_ordinal) as tr:
        stats = torch.zeros((batch, 4), dtype=torch.float32, device=tr.device)
        acc = torch.zeros(4, dtype=torch.float64, device=tr.device)
        since = 0
        t0 = time.time()
        for step in range(steps):
            idx = torch.randint(0, n, (batch,), generator=gen, device=tr.device)
            rate = lr * 0.5 * (1.0 + math.cos(math.pi * step / steps))
            soft = soft_targets(data["regret"][idx], temperature) if temperature > 0 else None
            tr.step(data["tiles"], data["tile_index"][idx], data["log2d"][idx], data["label_class"][idx],
                    data["label_qf"][idx], qf_weight, rate, stats, soft)
            acc += stats.double().mean(dim=0)
            since += 1
            if (step + 1) % 200 == 0 or step + 1 == steps:
                a = (acc / since).cpu().numpy()
                curve.append({"step": step + 1, "ce": float(a[0]), "qf_mse": float(a[1]), "accuracy": float(a[2])})
                log(f"step {step + 1}: ce {a[0]:.4f} qf_mse {a[1]:.4f} acc {a[2]:.4f} "
                    f"({time.time() - t0:.1f} s)")
                acc.zero_()
                since = 0
        params = tr.params()
    return params, norm, curve


def _bpp_psnr(nv12, w: int, h: int, d: float, net=None, margin: float = DEFAULT_MARGIN, flags: int = SPLIT):
    from . import Encoder
    from .decode import psnr_y
    with Encoder(w, h, d) as enc:
        if net is not None:
            enc.set_acsnet(net, margin, flags)
        data = enc.encode_host(nv12)
        decided = enc.acsnet_stats()[0] if net is not None else 0
        enc.set_acsnet(None)
    return 8.0 * len(data) / (w * h), psnr_y(nv12, data), decided


def codec_report(net: AcsNet, frames: list[tuple[int, int, int]], distances=(1.0, 2.0),
                 margin: float = DEFAULT_MARGIN, flags: int = SPLIT) -> list[dict]:
    """bpp and PSNR-Y of the learned-decision encode against the plain RD
    heuristic, per frame and distance, and the learned path's bpp change at
    the heuristic's PSNR-Y (log-bpp interpolated over distances d x 0.8..1.25)."""
    from .synth import make_nv12
    rows = []
    scales = (0.8, 0.9, 1.0, 1.12, 1.25)
    for (w, h, seed) in frames:
        nv12 = make_nv12(w, h, seed)
        for d in distances:
            bp, pp, _ = _bpp_psnr(nv12, w, h, d)
            curve = [_bpp_psnr(nv12, w, h, d * s, net, margin, flags) for s in scales]
            bl, pl, dec = curve[scales.index(1.0)]
            ps = np.array([c[1] for c in curve])
            lb = np.log(np.array([c[0] for c in curve]))
            order = np.argsort(ps)
            at = float(np.exp(np.interp(pp, ps[order], lb[order]))) if ps.min() <= pp <= ps.max() else float("nan")
            rows.append({"frame": f"{w}x{h}#{seed}", "distance": d, "bpp_plain": bp, "psnr_plain": pp,
                         "bpp_learned": bl, "psnr_learned": pl, "decided_regions": dec,
                         "regions": (w // 32) * (h // 32),
                         "bpp_delta_pct": 100.0 * (bl / bp - 1.0), "psnr_delta_db": pl - pp,
                         "bpp_delta_at_equal_psnr_pct": 100.0 * (at / bp - 1.0)})
    return rows


def _frames(n1080: int, n4k: int, seed0: int) -> list[tuple[int, int, int]]:
    return [(1920, 1080, seed0 + i) for i in range(n1080)] + [(3840, 2160, seed0 + 1000 + i) for i in range(n4k)]


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default=str(DEFAULT_WEIGHTS))
    ap.add_argument("--frames-1080p", type=int, default=48)
    ap.add_argument("--frames-4k", type=int, default=24)
    ap.add_argument("--val-frames", type=int, default=4)
    ap.add_argument("--distances", default="0.5,1,1.5,2,3,4")
    ap.add_argument("--steps", type=int, default=40000)
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--qf-weight", type=float, default=1.0)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--temperature", type=float, default=0.03)
    a = ap.parse_args(argv)
    dists = [float(x) for x in a.distances.split(",")]
    t0 = time.time()
    train_data = build_dataset(_frames(a.frames_1080p, a.frames_4k, 100), dists)
    val_data = build_dataset(_frames(a.val_frames, a.val_frames // 2, 50000), dists)
    t_data = time.time() - t0
    t1 = time.time()
    params, norm, curve = train(train_data, steps=a.steps, batch=a.batch, lr=a.lr, qf_weight=a.qf_weight,
                                seed=a.seed, temperature=a.temperature)
    t_train = time.time() - t1
    report = {"frames_1080p": a.frames_1080p, "frames_4k": a.frames_4k, "distances": dists,
              "train_samples": int(train_data["tile_index"].numel()),
              "train_tiles": int(train_data["tiles"].shape[0]), "steps": a.steps, "batch": a.batch,
              "lr": a.lr, "qf_weight": a.qf_weight, "seed": a.seed, "temperature": a.temperature,
              "dataset_seconds": round(t_data, 1),
              "train_seconds": round(t_train, 1), "curve": curve}
    with Trainer(params, norm, a.batch) as tr:
        report["train_eval"] = evaluate(tr, train_data)
        report["val_eval"] = evaluate(tr, val_data)
    with Trainer(init_params(a.seed), norm, a.batch) as tr:
        report["untrained_val_eval"] = evaluate(tr, val_data)
    out = Path(a.out)
    out.parent.mkdir(parents=True, exist_ok=True)
    out.write_bytes(pack_blob(params, norm))
    net = AcsNet(out.read_bytes())
    held_out = [(1920, 1080, 424242), (3840, 2160, 0)]
    report["codec_split"] = codec_report(net, held_out, flags=SPLIT)
    report["codec_split_qf"] = codec_report(net, held_out, flags=SPLIT | QF)
    net.close()
    out.with_suffix(".json").write_text(json.dumps(report, indent=1) + "\n")
    print(json.dumps({k: v for k, v in report.items() if k != "curve"}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
