"""ORACLE — test infrastructure only.

NumPy restatement of the coarse-grid corrector's network (3x3 "same"
convolutions, zero padding, GELU, MSE loss) in float64, with the device's
BF16 storage emulated by rounding to nearest even at the same places (inputs,
weights, inter-layer activations, gradients between layers).  Used by tests/
to check the device kernels' forward outputs and gradients, never by the
product.

Layouts follow include/claw_nn.h: activations NHWC [n][h][w][c], weights
[cout][9][cin] with tap = 3*ky + kx for the offset (ky-1, kx-1).
"""
from __future__ import annotations

import numpy as np


def bf16(a):
    """Round float32 values to BF16 (nearest even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def _shift(x, dy, dx):
    """x[n, y+dy, x+dx, c] with zeros outside."""
    n, h, w, c = x.shape
    out = np.zeros_like(x)
    ys, ye = max(0, -dy), min(h, h - dy)
    xs, xe = max(0, -dx), min(w, w - dx)
    out[:, ys:ye, xs:xe] = x[:, ys + dy:ye + dy, xs + dx:xe + dx]
    return out


def conv3x3(x, w, b=None):
    """y[n,y,x,co] = b[co] + sum_{tap,ci} w[co,tap,ci] x[n, y+ky-1, x+kx-1, ci]."""
    y = np.zeros(x.shape[:3] + (w.shape[0],))
    for tap in range(9):
        ky, kx = divmod(tap, 3)
        y += np.einsum("nhwc,oc->nhwo", _shift(x, ky - 1, kx - 1), w[:, tap, :])
    if b is not None:
        y += b
    return y


def conv3x3_wgrad(x, dz):
    """dw[co,tap,ci] = sum_p dz[p,co] x[p+off(tap),ci]; db[co] = sum_p dz[p,co]."""
    dw = np.zeros((dz.shape[-1], 9, x.shape[-1]))
    for tap in range(9):
        ky, kx = divmod(tap, 3)
        dw[:, tap, :] = np.einsum("nhwo,nhwc->oc", dz, _shift(x, ky - 1, kx - 1))
    return dw, dz.sum(axis=(0, 1, 2))


def flip(w):
    """wt[ci, tap, co] = w[co, 8 - tap, ci]: dx = conv3x3(dz, wt)."""
    return np.transpose(w[:, ::-1, :], (2, 1, 0))


GELU_K0 = np.sqrt(2.0 / np.pi)
GELU_K1 = 0.044715


def gelu(z):
    """GELU in its tanh form (Hendrycks and Gimpel 2016), as the device
    computes it: z/2 (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))."""
    return 0.5 * z * (1.0 + np.tanh(GELU_K0 * (z + GELU_K1 * z ** 3)))


def gelu_grad(z):
    t = np.tanh(GELU_K0 * (z + GELU_K1 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_K0 * (1.0 + 3.0 * GELU_K1 * z * z)


def forward(x, layers):
    """layers: [(w, b, act)]; returns the output and the per-layer
    (input, pre-activation) needed by backward.  Hidden activations are
    rounded to BF16 as the device stores them; the last layer's output stays
    float (the device writes it in FP32)."""
    cache = []
    a = bf16(x)
    for k, (w, b, act) in enumerate(layers):
        z = conv3x3(a, bf16(w), b)
        cache.append((a, z))
        if act:
            a = bf16(gelu(z))
        else:
            a = z
    return a, cache


def backward(dy, layers, cache):
    """Gradients of every layer's (w, b) for the output gradient dy, with the
    device's BF16 rounding of the propagated gradients."""
    grads = [None] * len(layers)
    d = bf16(dy)
    for k in range(len(layers) - 1, -1, -1):
        w, b, act = layers[k]
        a_in, z = cache[k]
        dz = bf16(d * gelu_grad(z)) if act else d
        grads[k] = conv3x3_wgrad(a_in, dz)
        if k > 0:
            d = bf16(conv3x3(dz, flip(bf16(w))))
    return grads


def mse_grad(pred, target):
    """Loss sum of squares over the first target channels and its gradient
    2 (pred - target) / count on them (zero on padding channels)."""
    nc = target.shape[-1]
    d = pred[..., :nc] - target
    g = np.zeros_like(pred)
    g[..., :nc] = 2.0 * d / d.size
    return float((d * d).sum()), g
