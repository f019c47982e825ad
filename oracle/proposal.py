"""ORACLE — test infrastructure only.

The learned seed proposal network restated in numpy, forward and backward,
as the checker of the device's BF16 tensor-core kernels
(semper-dic-engine_b200/csrc/kernels/proposal.cu). Imported only by tests.

Network (the task's proposal network): two 64x64 patches, stacked as two
input channels; five 3x3 convolutions of stride 2 and padding 1 with 16, 32,
64, 128 and 128 output channels, each followed by ReLU (64 -> 2 pixels a
side); the 128x2x2 features flattened; a 2-layer MLP, 512 -> 128 (ReLU) -> 6.
The six outputs are the affine map of patch coordinates (centred, in patch
pixels) from the first patch to the second: A = I + [[o0, o1], [o2, o3]] and
t = 16 * (o4, o5).

Arithmetic, as on the device: activations, weights and back-propagated
gradients enter every product as bfloat16 (round to nearest even); products
and sums are FP32; bias, ReLU and the loss in FP32; weights kept in FP32 and
rounded to bfloat16 for use. Layouts: activations NHWC, convolution weights
[co][kh][kw][ci], im2col columns ordered (kh, kw, ci). Every function follows
the dtype of its inputs (float64 inputs with bf16 replaced by the identity
give the exact gradients a finite-difference check needs).
"""
from __future__ import annotations

import numpy as np

CHANNELS = [2, 16, 32, 64, 128, 128]
FC = [512, 128, 6]
T_SCALE = 16.0
# loss points: a 3x3 grid over the patch, in patch pixels from its centre
LOSS_PTS = np.array([(x, y) for y in (-24.0, 0.0, 24.0) for x in (-24.0, 0.0, 24.0)], np.float32)


def bf16(a):
    """Round float32 to the nearest bfloat16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def init_params(seed=0):
    """He-normal weights, zero biases (FP32 masters)."""
    rng = np.random.default_rng(seed)
    p = {}
    for l in range(5):
        ci, co = CHANNELS[l], CHANNELS[l + 1]
        p[f"w{l}"] = (rng.standard_normal((co, 3, 3, ci)) * np.sqrt(2.0 / (9 * ci))).astype(np.float32)
        p[f"b{l}"] = np.zeros(co, np.float32)
    p["w5"] = (rng.standard_normal((FC[1], FC[0])) * np.sqrt(2.0 / FC[0])).astype(np.float32)
    p["b5"] = np.zeros(FC[1], np.float32)
    p["w6"] = (rng.standard_normal((FC[2], FC[1])) * np.sqrt(1.0 / FC[1]) * 0.1).astype(np.float32)
    p["b6"] = np.zeros(FC[2], np.float32)
    return p


def im2col(x):
    """x: [B, H, W, C] -> [B * H/2 * W/2, 9 * C], columns (kh, kw, c), zero padding."""
    B, H, W, C = x.shape
    xp = np.zeros((B, H + 2, W + 2, C), x.dtype)
    xp[:, 1:-1, 1:-1] = x
    Ho, Wo = H // 2, W // 2
    cols = np.zeros((B, Ho, Wo, 3, 3, C), x.dtype)
    for kh in range(3):
        for kw in range(3):
            cols[:, :, :, kh, kw] = xp[:, kh:kh + 2 * Ho:2, kw:kw + 2 * Wo:2]
    return cols.reshape(B * Ho * Wo, 9 * C)


def col2im(dcol, shape):
    """The adjoint of im2col: [B*Ho*Wo, 9C] -> [B, H, W, C]."""
    B, H, W, C = shape
    Ho, Wo = H // 2, W // 2
    d = dcol.reshape(B, Ho, Wo, 3, 3, C)
    dxp = np.zeros((B, H + 2, W + 2, C), dcol.dtype)
    for kh in range(3):
        for kw in range(3):
            dxp[:, kh:kh + 2 * Ho:2, kw:kw + 2 * Wo:2] += d[:, :, :, kh, kw]
    return dxp[:, 1:-1, 1:-1]


def forward(p, x):
    """x: [B, 64, 64, 2] (patch values, already normalised). Returns (out [B, 6], cache)."""
    cache = {"a": [bf16(x)]}
    a = cache["a"][0]
    for l in range(5):
        col = im2col(a)
        w = bf16(p[f"w{l}"].reshape(CHANNELS[l + 1], -1))
        y = col @ w.T + p[f"b{l}"]
        B, H, W, _ = a.shape
        a = bf16(np.maximum(y, 0.0)).reshape(B, H // 2, W // 2, CHANNELS[l + 1])
        cache["a"].append(a)
    f = a.reshape(a.shape[0], -1)  # (h, w, c) order of NHWC
    h = bf16(np.maximum(f @ bf16(p["w5"]).T + p["b5"], 0.0))
    cache["f"], cache["h"] = f, h
    out = h @ bf16(p["w6"]).T + p["b6"]
    return out, cache


def affine_of(out):
    """(A [B, 2, 2], t [B, 2]) from the six outputs."""
    A = np.zeros((out.shape[0], 2, 2), np.float64)
    A[:, 0, 0] = 1.0 + out[:, 0]
    A[:, 0, 1] = out[:, 1]
    A[:, 1, 0] = out[:, 2]
    A[:, 1, 1] = 1.0 + out[:, 3]
    return A, T_SCALE * np.asarray(out[:, 4:6], np.float64)


def loss_and_grad(out, target):
    """Mean over the batch and the loss points of the squared displacement
    error of the predicted affine map (patch pixels^2), and d loss / d out."""
    d = out - target
    B = out.shape[0]
    P = LOSS_PTS
    ex = d[:, 0:1] * P[None, :, 0] + d[:, 1:2] * P[None, :, 1] + T_SCALE * d[:, 4:5]
    ey = d[:, 2:3] * P[None, :, 0] + d[:, 3:4] * P[None, :, 1] + T_SCALE * d[:, 5:6]
    n = B * len(P)
    loss = float((ex ** 2 + ey ** 2).sum() / n)
    g = np.zeros_like(d)
    g[:, 0] = (2 * ex * P[None, :, 0]).sum(1) / n
    g[:, 1] = (2 * ex * P[None, :, 1]).sum(1) / n
    g[:, 4] = (2 * ex * T_SCALE).sum(1) / n
    g[:, 2] = (2 * ey * P[None, :, 0]).sum(1) / n
    g[:, 3] = (2 * ey * P[None, :, 1]).sum(1) / n
    g[:, 5] = (2 * ey * T_SCALE).sum(1) / n
    return loss, g


def backward(p, cache, gout):
    """Gradients of every parameter given d loss / d out."""
    g = {}
    h, f = cache["h"], cache["f"]
    go = bf16(gout)
    g["w6"] = go.T @ h
    g["b6"] = gout.sum(0)
    dh = go @ bf16(p["w6"])
    dh = np.where(h > 0, dh, 0.0)
    dhb = bf16(dh)
    g["w5"] = dhb.T @ f
    g["b5"] = dh.sum(0)
    df = dhb @ bf16(p["w5"])
    a = cache["a"]
    da = df.reshape(a[5].shape)
    for l in range(4, -1, -1):
        dy = np.where(a[l + 1] > 0, da, 0.0)
        B, Ho, Wo, Co = dy.shape
        dy2 = dy.reshape(-1, Co)
        dyb = bf16(dy2)
        col = im2col(a[l])
        g[f"w{l}"] = (dyb.T @ col).reshape(Co, 3, 3, CHANNELS[l])
        g[f"b{l}"] = dy2.sum(0)
        if l > 0:
            dcol = dyb @ bf16(p[f"w{l}"].reshape(Co, -1))
            da = col2im(dcol, a[l].shape)
    return g


def param_names():
    return [n for l in range(7) for n in (f"w{l}", f"b{l}")]


def flatten(p):
    """The flat parameter vector of the device (w0 b0 ... w6 b6)."""
    return np.concatenate([np.asarray(p[n], np.float32).ravel() for n in param_names()])


def unflatten(flat):
    shapes = {}
    for l in range(5):
        shapes[f"w{l}"] = (CHANNELS[l + 1], 3, 3, CHANNELS[l])
        shapes[f"b{l}"] = (CHANNELS[l + 1],)
    shapes["w5"], shapes["b5"] = (FC[1], FC[0]), (FC[1],)
    shapes["w6"], shapes["b6"] = (FC[2], FC[1]), (FC[2],)
    p, o = {}, 0
    for n in param_names():
        k = int(np.prod(shapes[n]))
        p[n] = np.asarray(flat[o:o + k], np.float32).reshape(shapes[n])
        o += k
    assert o == len(flat)
    return p
