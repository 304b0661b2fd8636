"""CPU oracle of the transform-decision network. Test infrastructure only:
imported by tests/ as the checker, never on the product path.

The network has no counterpart in the reference: it is one of the
non-reference forms (learned transform and quant-field decisions) built next
to the drop-in path. This file restates its arithmetic in numpy so that the
CUDA forward, loss and gradients can be checked:

  * forward: im2col matrices times the weight matrices, in float64, with the
    values rounded to float32 and then BF16 (nearest, ties to even) at the
    points where the kernels round: the normalised input, every post-ReLU
    activation, the loss gradient at the outputs and every masked data
    gradient;
  * backward: the textbook im2col / col2im formulation (the kernels use a
    gather per input pixel instead, so the two are independent);
  * with rounding switched off the same code is plain float64 calculus, which
    the tests pin against central finite differences of the loss.

Parity of the CUDA kernels against this oracle is approximate by nature (the
tensor cores accumulate in their own order and a BF16 rounding boundary can
fall between the two): outputs and gradients are compared by relative L2
error with the tolerance written in each test.
"""

from __future__ import annotations

import numpy as np

C = 32
NIN = 8
NCLS = 17
K1 = 80
K = 288
OFF_W = (0, C * K1, C * K1 + C * K, C * K1 + 2 * C * K)
NW = C * K1 + 3 * C * K  # 30208
OFF_B = NW
NPARAMS = NW + 4 * C     # 30336
KS = (K1, K, K, K)


def bf16(x) -> np.ndarray:
    """float32 -> BF16 (round to nearest, ties to even), returned as float32."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16).astype(np.uint32)
    out = r.view(np.float32).copy()
    out[np.isnan(a)] = np.nan
    return out


def weights(params: np.ndarray, layer: int, rnd: bool = True) -> np.ndarray:
    w = np.asarray(params[OFF_W[layer]:OFF_W[layer] + C * KS[layer]], np.float32).reshape(C, KS[layer])
    return (bf16(w) if rnd else w).astype(np.float64)


def biases(params: np.ndarray, layer: int) -> np.ndarray:
    return np.asarray(params[OFF_B + layer * C:OFF_B + (layer + 1) * C], np.float32).astype(np.float64)


def im2col(x: np.ndarray, stride: int, pad: int = 1) -> np.ndarray:
    """[H][W][Cin] -> [P][9 Cin], column = (ky * 3 + kx) * Cin + ci, zero padding `pad`."""
    h, w, cn = x.shape
    oh, ow = (h + 2 * pad - 3) // stride + 1, (w + 2 * pad - 3) // stride + 1
    xp = np.zeros((h + 2 * pad, w + 2 * pad, cn), np.float64)
    xp[pad:pad + h, pad:pad + w] = x
    cols = [xp[ky:ky + stride * oh:stride, kx:kx + stride * ow:stride, :] for ky in range(3) for kx in range(3)]
    return np.concatenate(cols, axis=2).reshape(oh * ow, 9 * cn)


def col2im(dcol: np.ndarray, h: int, stride: int, cn: int) -> np.ndarray:
    """Adjoint of im2col with padding 1: [P][9 Cin] -> [H][W][Cin]."""
    oh = (h - 1) // stride + 1
    d = dcol[:, :9 * cn].reshape(oh, oh, 9, cn)
    dxp = np.zeros((h + 2, h + 2, cn), np.float64)
    for ky in range(3):
        for kx in range(3):
            dxp[ky:ky + stride * oh:stride, kx:kx + stride * oh:stride, :] += d[:, :, ky * 3 + kx, :]
    return dxp[1:-1, 1:-1]


def _r(v: np.ndarray, rnd: bool) -> np.ndarray:
    return bf16(np.asarray(v, np.float32)).astype(np.float64) if rnd else np.asarray(v, np.float64)


def net_input(norm: np.ndarray, tile: np.ndarray, log2d: float, rnd: bool = True) -> np.ndarray:
    """[3][34][34] XYB tile (a region and its 1-pixel ring) -> [34][34][8]
    input (X, Y, B, log2 distance, zeros)."""
    scale = np.asarray(norm[:4], np.float32)
    shift = np.asarray(norm[4:8], np.float32)
    x = np.zeros((34, 34, NIN), np.float64)
    for c in range(3):
        v = (np.asarray(tile[c], np.float32) - shift[c]) * scale[c] if rnd else \
            (np.asarray(tile[c], np.float64) - float(shift[c])) * float(scale[c])
        x[:, :, c] = _r(v, rnd)
    v = (np.float32(log2d) - shift[3]) * scale[3] if rnd else (float(log2d) - float(shift[3])) * float(scale[3])
    x[:, :, 3] = _r(np.full((34, 34), v), rnd)
    return x


PADS = (0, 1, 1, 1)
STRIDES = (2, 2, 2, 1)


def _layer(x: np.ndarray, params: np.ndarray, layer: int, relu: bool, rnd: bool):
    a = im2col(x, STRIDES[layer], PADS[layer])
    if a.shape[1] < KS[layer]:
        a = np.pad(a, ((0, 0), (0, KS[layer] - a.shape[1])))
    y = a @ weights(params, layer, rnd).T + biases(params, layer)
    if not relu:
        return np.asarray(y, np.float32).astype(np.float64) if rnd else y
    return _r(np.maximum(y, 0.0), rnd)


def forward(params: np.ndarray, norm: np.ndarray, tile: np.ndarray, log2d: float, rnd: bool = True) -> dict:
    """Activations x1 [34,34,8], x2 [16,16,32], x3 [8,8,32], x4 [4,4,32] and out [16][32]."""
    x1 = net_input(norm, tile, log2d, rnd)
    x2 = _layer(x1, params, 0, True, rnd).reshape(16, 16, C)
    x3 = _layer(x2, params, 1, True, rnd).reshape(8, 8, C)
    x4 = _layer(x3, params, 2, True, rnd).reshape(4, 4, C)
    out = _layer(x4, params, 3, False, rnd)
    return {"x1": x1, "x2": x2, "x3": x3, "x4": x4, "out": out}


def head(out: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(17 split logits, 16 log2 quant fields) from the [16][32] outputs."""
    return out[:, 1:1 + NCLS].sum(axis=0) * 0.0625, out[:, 0].copy()


def softmax_stats(logits: np.ndarray) -> tuple[np.ndarray, int, float, float]:
    """(probabilities, arg-max, top-two margin, log-sum-exp)."""
    m = float(np.max(logits))
    e = np.exp(logits - m)
    s = float(e.sum())
    top = int(np.argmax(logits))
    second = float(np.max(np.delete(e, top)))
    return e / s, top, (float(e[top]) - second) / s, float(np.log(s) + m)


def decide(out: np.ndarray, margin: float) -> tuple[int, np.ndarray]:
    """Inference decision of one region: class or -1, and the 16 quant fields."""
    logits, qf = head(out)
    _, top, mg, _ = softmax_stats(logits)
    q = np.clip(np.rint(np.exp2(qf)), 1, 256).astype(np.int32)
    return (top if mg >= margin else -1), q


def loss_and_grad(params: np.ndarray, norm: np.ndarray, tiles: np.ndarray, log2d: np.ndarray,
                  labels: np.ndarray, label_qf: np.ndarray, qf_weight: float, rnd: bool = True,
                  soft: np.ndarray | None = None):
    """Mean loss over the batch, per-sample stats [n][4] and the gradient
    [NPARAMS]; `soft` [n][17] replaces the one-hot split targets."""
    n = len(tiles)
    grad = np.zeros(NPARAMS, np.float64)
    stats = np.zeros((n, 4), np.float64)
    total = 0.0
    w = [weights(params, l, rnd) for l in range(4)]
    for i in range(n):
        f = forward(params, norm, tiles[i], float(log2d[i]), rnd)
        logits, qf = head(f["out"])
        prob, top, mg, lse = softmax_stats(logits)
        lab = int(labels[i])
        target = np.eye(NCLS)[lab] if soft is None else np.asarray(soft[i], np.float64)
        ce = lse - float((target * logits).sum())
        d = qf - np.asarray(label_qf[i], np.float64)
        sq = float((d * d).sum())
        stats[i] = (ce, sq / 16.0, 1.0 if top == lab else 0.0, mg)
        total += ce + qf_weight * sq / 16.0
        dlogit = (prob - target) / n
        g = np.zeros((16, C), np.float64)
        g[:, 0] = 2.0 * qf_weight * d / n / 16.0
        g[:, 1:1 + NCLS] = dlogit[None, :] / 16.0
        g = _r(g, rnd)
        xs = [f["x1"], f["x2"], f["x3"], f["x4"]]
        for layer in (3, 2, 1, 0):
            a = im2col(xs[layer], STRIDES[layer], PADS[layer])
            if a.shape[1] < KS[layer]:
                a = np.pad(a, ((0, 0), (0, KS[layer] - a.shape[1])))
            grad[OFF_W[layer]:OFF_W[layer] + C * KS[layer]] += (g.T @ a).reshape(-1)
            grad[OFF_B + layer * C:OFF_B + (layer + 1) * C] += g.sum(axis=0)
            if layer == 0:
                break
            h = xs[layer].shape[0]
            dx = col2im(g @ w[layer], h, STRIDES[layer], C)
            g = _r(np.where(xs[layer] > 0, dx, 0.0), rnd).reshape(h * h, C)
    return total / n, stats, grad


def split_class(acs: np.ndarray) -> int:
    """Split class of a full region from its 4x4 block AC strategy (side at
    first blocks, 0 at covered blocks), or -1 if it is not a region split."""
    if acs[0, 0] == 32:
        return 0
    m = 0
    for q in range(4):
        qy, qx = q >> 1, q & 1
        s = int(acs[2 * qy, 2 * qx])
        if s == 8:
            m |= 1 << q
        elif s != 16:
            return -1
    return 1 + m
