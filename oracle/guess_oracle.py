"""CPU restatement of the learned starting guess for the departure-point
iteration.  TEST INFRASTRUCTURE ONLY: the product path never imports this
module; tests, smoke() and the bench's CPU leg use it as the checker.

The reference has no learned guess: its trajectory starts from the previous
step's departure points, or from the arrival point on the first step
(src/gemdyn/src/base/adz_traject.F90:60-112, adz_inittraj.F90).  The network
and its training are this project's own; what this module pins is the
arithmetic the CUDA kernels must reproduce:

features   for arrival point (i, j, k) the prepared departure winds
           (adz_prepareWinds.F90:40-97: u*cy/rayt, v/rayt and w on momentum
           levels) at the 27 points (i+di, j+dj, k+dk), dk outer, di inner,
           k+dk clamped to 1..nk, as Courant numbers
               u dt / hx,  v dt / hy,  w dt / dz(nb),  nb = min(max(k,1),nk-1)
           (dz from the 1/dz table of the momentum levels), then dt / 300 s:
           82 values.
network    y = W3 g(W2 g(W1 x + b1) + b2) + b3, 82 -> 128 -> 128 -> 3, with
           g the tanh form of GELU, 0.5 x (1 + tanh(sqrt(2/pi)(x + 0.044715 x^3)))
           (Hendrycks and Gimpel, 2016).
target     the departure displacement in grid indices,
               (i + i0g - 1 - x_dep,  j + j0g - 1 - y_dep,  k - z_dep),
           of the converged plain iteration.
inference  BF16 weights and BF16 layer inputs, FP32 accumulation and FP32
           bias + GELU (forward_bf16).
training   mean squared error over the three components, backward pass in
           FP32 (backward), Adam (adam_step).
"""
from __future__ import annotations

import numpy as np

NFEAT = 82
HID = 128
NOUT = 3
DT_SCALE = 300.0
_C = np.sqrt(2.0 / np.pi)


def gelu(x):
    x = np.asarray(x, np.float32)
    return (0.5 * x * (1.0 + np.tanh(np.float32(_C) * (x + np.float32(0.044715) * x * x * x)))).astype(np.float32)


def gelu_grad(x):
    x = np.asarray(x, np.float64)
    u = _C * (x + 0.044715 * x ** 3)
    t = np.tanh(u)
    du = _C * (1.0 + 3 * 0.044715 * x * x)
    return (0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * du).astype(np.float32)


def bf16(a):
    """Round to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out).astype(np.float32)


def init_params(seed=0):
    """He-style initialisation; the same draw seeds the CUDA trainer."""
    rng = np.random.default_rng(seed)
    p = {}
    for name, (n, k) in {"1": (HID, NFEAT), "2": (HID, HID), "3": (NOUT, HID)}.items():
        p["W" + name] = (rng.standard_normal((n, k)) * np.sqrt(2.0 / k)).astype(np.float32)
        p["b" + name] = np.zeros(n, np.float32)
    p["W3"] *= np.float32(0.1)
    return p


def forward(p, x):
    """FP32 forward pass; returns (y, cache)."""
    x = np.asarray(x, np.float32)
    h1 = x @ p["W1"].T + p["b1"]
    a1 = gelu(h1)
    h2 = a1 @ p["W2"].T + p["b2"]
    a2 = gelu(h2)
    y = a2 @ p["W3"].T + p["b3"]
    return y.astype(np.float32), (x, h1, a1, h2, a2)


def forward_bf16(p, x):
    """Inference arithmetic: BF16 weights and layer inputs, FP32 sums."""
    a0 = bf16(x)
    h1 = (a0.astype(np.float64) @ bf16(p["W1"]).T.astype(np.float64)).astype(np.float32) + p["b1"]
    a1 = bf16(gelu(h1))
    h2 = (a1.astype(np.float64) @ bf16(p["W2"]).T.astype(np.float64)).astype(np.float32) + p["b2"]
    a2 = bf16(gelu(h2))
    y = (a2.astype(np.float64) @ bf16(p["W3"]).T.astype(np.float64)).astype(np.float32) + p["b3"]
    return y.astype(np.float32)


def loss(p, x, t):
    y, _ = forward(p, x)
    d = y.astype(np.float64) - t
    return float(np.mean(np.sum(d * d, axis=1)))


def backward(p, x, t):
    """Gradients of mean_b sum_c (y - t)^2 with respect to every parameter."""
    y, (x, h1, a1, h2, a2) = forward(p, x)
    B = x.shape[0]
    dy = (2.0 / B) * (y - t).astype(np.float32)
    g = {"W3": dy.T @ a2, "b3": dy.sum(0)}
    da2 = dy @ p["W3"]
    dh2 = da2 * gelu_grad(h2)
    g["W2"], g["b2"] = dh2.T @ a1, dh2.sum(0)
    da1 = dh2 @ p["W2"]
    dh1 = da1 * gelu_grad(h1)
    g["W1"], g["b1"] = dh1.T @ x, dh1.sum(0)
    return {k: v.astype(np.float32) for k, v in g.items()}


def adam_step(p, m, v, g, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update in place (Kingma and Ba, 2015), bias-corrected."""
    c1 = 1.0 - b1 ** step
    c2 = 1.0 - b2 ** step
    for k in p:
        m[k] = (b1 * m[k] + (1 - b1) * g[k]).astype(np.float32)
        v[k] = (b2 * v[k] + (1 - b2) * g[k] * g[k]).astype(np.float32)
        p[k] = (p[k] - lr * (m[k] / c1) / (np.sqrt(v[k] / c2) + eps)).astype(np.float32)


def features(uvw, nit, njt, nk, halo, ni, nj, k00, dt, inv_hx, inv_hy, odelz_m):
    """Features of every arrival point (i 1..ni, j 1..nj, k k00..nk), in the
    order k, j, i (i fastest).  uvw: prepared departure winds as three planes
    (3, nk, njt, nit) of the ext layout (1-halo : n+halo, ..., 1:nk)."""
    u = np.asarray(uvw, np.float64)
    kk = np.arange(k00, nk + 1)
    jj = np.arange(1, nj + 1)
    ii = np.arange(1, ni + 1)
    nb = np.clip(kk, 1, nk - 1)
    sz = (dt * np.asarray(odelz_m, np.float64)[nb])[:, None, None]
    out = np.empty((len(kk), nj, ni, NFEAT), np.float32)
    n = 0
    for dk in (-1, 0, 1):
        kq = np.clip(kk + dk, 1, nk) - 1
        for dj in (-1, 0, 1):
            jq = jj + dj - 1 + halo
            for di in (-1, 0, 1):
                iq = ii + di - 1 + halo
                blk = u[:, kq][:, :, jq][:, :, :, iq]
                out[..., 3 * n + 0] = (blk[0] * dt * inv_hx).astype(np.float32)
                out[..., 3 * n + 1] = (blk[1] * dt * inv_hy).astype(np.float32)
                out[..., 3 * n + 2] = (blk[2] * sz).astype(np.float32)
                n += 1
    out[..., 81] = np.float32(dt / DT_SCALE)
    return out.reshape(-1, NFEAT)
