"""ORACLE - test infrastructure only.  A numpy restatement of the proposal
network's forward pass and its gradients, used by tests/ as the checker of
the tensor-core kernels.  The product never imports it.

The network has no counterpart in the reference, so parity is pinned in two
ways:
- by finite differences of this restatement in float64 (rounding off);
- against the device at the rounding points the device uses (rounding on).
  Weights are rounded to BF16 for the products, activations and
  pre-activation gradients are stored in BF16, and every sum is exact here
  (float64), where the device accumulates in FP32.

Layout: activations (batch, z, y, x, channels).  Conv weights
(cout, 27, cin) with tap = (kz * 3 + ky) * 3 + kx; output voxel o reads input
voxel o * stride + k - 1 (zero padding of one).
"""

from __future__ import annotations

import numpy as np

LAYERS = ((2, 16, 1), (16, 32, 2), (32, 64, 2), (64, 64, 2))  # (cin, cout, stride)


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    x = np.ascontiguousarray(x, np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return (b & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(x.shape)


def _taps():
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                yield (kz * 3 + ky) * 3 + kx, kz, ky, kx


def _tap_slice(xp, kz, ky, kx, stride, so):
    return xp[:, kz:kz + stride * so:stride, ky:ky + stride * so:stride, kx:kx + stride * so:stride, :]


def conv_forward(x, w, b, stride):
    """ReLU(conv(x, w) + b), sums in float64."""
    s = x.shape[1]
    so = s // stride
    xp = np.pad(x.astype(np.float64), ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((x.shape[0], so, so, so, w.shape[0]), np.float64)
    for tap, kz, ky, kx in _taps():
        out += np.einsum("bzyxc,oc->bzyxo", _tap_slice(xp, kz, ky, kx, stride, so), w[:, tap, :].astype(np.float64))
    out += b.astype(np.float64)
    return np.maximum(out, 0.0)


def conv_weight_grad(x, dy, stride):
    """dW (cout, 27, cin) and db (cout,) of conv(x) for output gradient dy."""
    so = dy.shape[1]
    xp = np.pad(x.astype(np.float64), ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    dyd = dy.astype(np.float64)
    dw = np.zeros((dy.shape[-1], 27, x.shape[-1]), np.float64)
    for tap, kz, ky, kx in _taps():
        dw[:, tap, :] = np.einsum("bzyxo,bzyxc->oc", dyd, _tap_slice(xp, kz, ky, kx, stride, so))
    return dw, dyd.sum(axis=(0, 1, 2, 3))


def conv_data_grad(dy, w, stride, s_in):
    """Gradient w.r.t. the conv input (batch, s_in^3, cin)."""
    so = dy.shape[1]
    dxp = np.zeros((dy.shape[0], s_in + 2, s_in + 2, s_in + 2, w.shape[2]), np.float64)
    dyd = dy.astype(np.float64)
    for tap, kz, ky, kx in _taps():
        dxp[:, kz:kz + stride * so:stride, ky:ky + stride * so:stride, kx:kx + stride * so:stride, :] += np.einsum(
            "bzyxo,oc->bzyxc", dyd, w[:, tap, :].astype(np.float64))
    return dxp[:, 1:-1, 1:-1, 1:-1, :]


def split(flat):
    """Parameter blocks of the flat vector: [(w, b) per layer], head_w, head_b."""
    flat = np.asarray(flat)
    layers, off = [], 0
    for cin, cout, _ in LAYERS:
        n = cout * 27 * cin
        w = flat[off:off + n].reshape(cout, 27, cin)
        off += n
        b = flat[off:off + cout]
        off += cout
        layers.append((w, b))
    head_w = flat[off:off + 64]
    head_b = flat[off + 64:off + 65]
    return layers, head_w, head_b


def forward(flat, x, rounding=True):
    """Predictions and the stored activations for inputs x (batch, s, s, s, 2)."""
    r = bf16 if rounding else (lambda v: np.asarray(v, np.float64))
    layers, head_w, head_b = split(flat)
    acts = [r(x)]
    for (w, b), (_, _, stride) in zip(layers, LAYERS):
        acts.append(r(conv_forward(acts[-1], r(w), b, stride)))
    last = acts[-1].astype(np.float64)
    pooled = last.mean(axis=(1, 2, 3))
    pred = pooled @ head_w.astype(np.float64) + float(head_b[0])
    return pred, acts, pooled


def gradients(flat, x, labels, rounding=True):
    """(loss, flat gradient) of the mean squared error."""
    r = bf16 if rounding else (lambda v: np.asarray(v, np.float64))
    layers, head_w, head_b = split(flat)
    pred, acts, pooled = forward(flat, x, rounding)
    y = np.asarray(labels, np.float64)
    batch = len(y)
    loss = float(np.mean((pred - y) ** 2))
    dpred = 2.0 * (pred - y) / batch
    g_head_w = dpred @ pooled
    g_head_b = np.array([dpred.sum()])
    last = acts[-1]
    voxels = last.shape[1] * last.shape[2] * last.shape[3]
    g = dpred[:, None] * head_w.astype(np.float64)[None, :] / voxels
    dpre = r(np.broadcast_to(g[:, None, None, None, :], last.shape) * (last > 0))
    grads = [None] * len(LAYERS)
    for i in range(len(LAYERS) - 1, -1, -1):
        w, _ = layers[i]
        stride = LAYERS[i][2]
        dw, db = conv_weight_grad(acts[i], dpre, stride)
        grads[i] = (dw, db)
        if i > 0:
            dx = conv_data_grad(dpre, r(w), stride, acts[i].shape[1])
            dpre = r(dx * (acts[i] > 0))
    flat_grad = []
    for dw, db in grads:
        flat_grad += [dw.ravel(), db.ravel()]
    flat_grad += [g_head_w.ravel(), g_head_b.ravel()]
    return loss, np.concatenate(flat_grad)


def he_parameters(seed, scale_head=0.125):
    """Float64 parameters for CPU checks (not the device's initialiser)."""
    rng = np.random.default_rng(seed)
    parts = []
    for cin, cout, _ in LAYERS:
        parts.append(rng.normal(0, np.sqrt(2.0 / (27 * cin)), cout * 27 * cin))
        parts.append(rng.normal(0, 0.05, cout))
    parts.append(rng.normal(0, scale_head, 64))
    parts.append(rng.normal(0, 0.05, 1))
    return np.concatenate(parts)
