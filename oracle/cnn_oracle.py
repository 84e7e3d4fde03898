"""TEST INFRASTRUCTURE ONLY: float64 numpy restatement of the correction CNN of
the learned narrow-kernel path (projects_b200/csrc/gridrec_cnn.cu), forward and
backward, used by the tests to check the device kernels' outputs and gradients.
Not part of the product.  The reference has no such network; this file states
the network's definition:

    h1 = relu(conv1(x)), h2 = relu(conv2(h1)), y = x + conv3(h2)
    conv(x)[p] = b + sum_tap w[tap] x[p + (dy, dx)],  tap = (dy + 1) * 3 + (dx + 1),
    zero padding; loss = mean (y - target)^2.

Parameter vector (float32 on the device, float64 here):
    w1[tap][co] (144), b1 (16), w2[tap][co][ci] (2304), b2 (16), w3[tap][ci] (144), b3 (1)
"""
from __future__ import annotations

import numpy as np

C = 16
OFF = {"w1": 0, "b1": 144, "w2": 160, "b2": 2464, "w3": 2480, "b3": 2624}
N_PARAMS = 2625


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[0:144].reshape(9, C), p[144:160], p[160:2464].reshape(9, C, C), p[2464:2480],
            p[2480:2624].reshape(9, C), p[2624])


def _shift(a, dy, dx):
    """out[y, x] = a[y + dy, x + dx] (zero outside); a: (N, H, W, ...)."""
    out = np.zeros_like(a)
    H, W = a.shape[1], a.shape[2]
    ys, yd = slice(max(dy, 0), H + min(dy, 0)), slice(max(-dy, 0), H + min(-dy, 0))
    xs, xd = slice(max(dx, 0), W + min(dx, 0)), slice(max(-dx, 0), W + min(-dx, 0))
    out[:, yd, xd] = a[:, ys, xs]
    return out


TAPS = [(t // 3 - 1, t % 3 - 1) for t in range(9)]


def forward(p, x, bf16=False, x_conv1=None):
    """x (N, H, W) -> dict of h1, h2 (N, H, W, 16), y (N, H, W).  bf16=True rounds the
    stored hidden activations to bfloat16 as the device does; x_conv1 (optional) is
    conv1's input in place of x (a rounded copy of it), the residual still adds x."""
    w1, b1, w2, b2, w3, b3 = unpack(p)
    x = np.asarray(x, np.float64)
    xc = x if x_conv1 is None else np.asarray(x_conv1, np.float64)
    rnd = _bf16 if bf16 else (lambda a: a)
    z1 = np.broadcast_to(b1, x.shape + (C,)).copy()
    for t, (dy, dx) in enumerate(TAPS):
        z1 += _shift(xc, dy, dx)[..., None] * w1[t]
    h1 = rnd(np.maximum(z1, 0.0))
    z2 = np.broadcast_to(b2, x.shape + (C,)).copy()
    for t, (dy, dx) in enumerate(TAPS):
        z2 += _shift(h1, dy, dx) @ w2[t].T
    h2 = rnd(np.maximum(z2, 0.0))
    y = x + b3
    for t, (dy, dx) in enumerate(TAPS):
        y = y + _shift(h2, dy, dx) @ w3[t]
    return {"h1": h1, "h2": h2, "y": y}


def loss_and_grads(p, x, target, bf16=False):
    """Mean-squared loss and its gradient with respect to the parameter vector."""
    w1, b1, w2, b2, w3, b3 = unpack(p)
    f = forward(p, x, bf16)
    x = np.asarray(x, np.float64)
    h1, h2, y = f["h1"], f["h2"], f["y"]
    n = y.size
    d = y - target
    loss = float((d * d).sum() / n)
    gy = 2.0 * d / n
    g = np.zeros(N_PARAMS)
    rnd = _bf16 if bf16 else (lambda a: a)
    # conv3
    g_h2 = np.zeros_like(h2)
    for t, (dy, dx) in enumerate(TAPS):
        g[OFF["w3"] + t * C:OFF["w3"] + (t + 1) * C] = (gy[..., None] * _shift(h2, dy, dx)).sum((0, 1, 2))
        g_h2 += _shift(gy, -dy, -dx)[..., None] * w3[t]
    g[OFF["b3"]] = gy.sum()
    gz2 = rnd(g_h2 * (h2 > 0))
    # conv2
    g_h1 = np.zeros_like(h1)
    for t, (dy, dx) in enumerate(TAPS):
        sh = _shift(h1, dy, dx)
        g[OFF["w2"] + t * C * C:OFF["w2"] + (t + 1) * C * C] = np.einsum(
            "nhwo,nhwi->oi", gz2, sh).ravel()
        g_h1 += _shift(gz2, -dy, -dx) @ w2[t]
    g[OFF["b2"]:OFF["b2"] + C] = gz2.sum((0, 1, 2))
    gz1 = rnd(g_h1 * (h1 > 0))
    # conv1
    for t, (dy, dx) in enumerate(TAPS):
        g[OFF["w1"] + t * C:OFF["w1"] + (t + 1) * C] = (gz1 * _shift(x, dy, dx)[..., None]).sum((0, 1, 2))
    g[OFF["b1"]:OFF["b1"] + C] = gz1.sum((0, 1, 2))
    return loss, g


def _bf16(a):
    """Round float64 values to bfloat16 (round to nearest even), back as float64."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64).reshape(np.shape(a))
