"""TEST INFRASTRUCTURE ONLY: CPU restatement of the closure MLP
(45 -> 64 -> 64 -> 2, tanh-form GELU, mean squared error) in FP64 numpy, for checking
the CUDA kernels of inmsom_elfs_b200/csrc/closure.cu.  It has no
counterpart in the reference (the closure is this project's addition).

emulate=True rounds to BF16 exactly where the kernels store BF16: the
inputs, the weights, the activations a1, a2 and the back-propagated
gradients d3, d2, d1 (bias gradients use the unrounded values)."""
from __future__ import annotations

import math

import numpy as np

KIN, HID, NOUT, N3 = 48, 64, 2, 8
OFF_W1 = 0
OFF_B1 = OFF_W1 + KIN * HID
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + HID * N3
NPARAM = OFF_B3 + N3

GC0 = math.sqrt(2.0 / math.pi)
GC1 = GC0 * 0.044715


def bf16(a):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    a32 = np.asarray(a, dtype=np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    """GELU in the tanh form (Hendrycks & Gimpel 2016), as the kernels use it."""
    return 0.5 * x * (1.0 + np.tanh(x * (GC0 + GC1 * x * x)))


def gelu_d(x):
    t = np.tanh(x * (GC0 + GC1 * x * x))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * (GC0 + 3.0 * GC1 * x * x)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(KIN, HID), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(HID, HID),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3].reshape(HID, N3), p[OFF_B3:NPARAM])


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform weights for the GELU layers, Glorot for the output,
    zero biases; padded rows/columns zero."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, dtype=np.float32)
    w1 = rng.uniform(-1, 1, (KIN, HID)) * math.sqrt(6.0 / 45)
    w1[45:] = 0.0
    w2 = rng.uniform(-1, 1, (HID, HID)) * math.sqrt(6.0 / HID)
    w3 = np.zeros((HID, N3))
    w3[:, :NOUT] = rng.uniform(-1, 1, (HID, NOUT)) * math.sqrt(6.0 / (HID + NOUT))
    p[OFF_W1:OFF_B1] = w1.ravel()
    p[OFF_W2:OFF_B2] = w2.ravel()
    p[OFF_W3:OFF_B3] = w3.ravel()
    return p


def forward(p, x, emulate=True):
    """x: [n, 48] -> (y [n, 2], cache)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    r = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
    x = r(x)
    W1, W2, W3 = r(W1), r(W2), r(W3)
    b1, b2, b3 = (np.asarray(b, dtype=np.float32).astype(np.float64) for b in (b1, b2, b3))
    z1 = x @ W1 + b1
    a1 = r(gelu(z1))
    z2 = a1 @ W2 + b2
    a2 = r(gelu(z2))
    z3 = a2 @ W3 + b3
    return z3[:, :NOUT], (x, z1, a1, z2, a2, z3, W1, W2, W3)


def loss_grad(p, x, t, emulate=True):
    """Mean squared error over the batch and its gradient (NPARAM)."""
    r = bf16 if emulate else (lambda a: np.asarray(a, dtype=np.float64))
    y, (x, z1, a1, z2, a2, z3, W1, W2, W3) = forward(p, x, emulate)
    n = x.shape[0]
    e = y - t
    loss = float(np.sum(e * e) / (n * NOUT))
    dz3 = np.zeros((n, N3))
    dz3[:, :NOUT] = 2.0 * e / (n * NOUT)
    d3 = r(dz3)
    g = np.zeros(NPARAM)
    g[OFF_W3:OFF_B3] = (a2.T @ d3).ravel()
    g[OFF_B3:NPARAM] = dz3.sum(0)
    dz2 = (d3 @ W3.T) * gelu_d(z2)
    d2 = r(dz2)
    g[OFF_W2:OFF_B2] = (a1.T @ d2).ravel()
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    dz1 = (d2 @ W2.T) * gelu_d(z1)
    d1 = r(dz1)
    g[OFF_W1:OFF_B1] = (x.T @ d1).ravel()
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    return loss, g


def adam(p, m, v, g, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One bias-corrected Adam step on the unpadded parameters."""
    p, m, v = p.copy(), m.copy(), v.copy()
    mask = np.ones(NPARAM, bool)
    mask[OFF_W1 + 45 * HID:OFF_B1] = False
    w3 = np.zeros((HID, N3), bool)
    w3[:, NOUT:] = True
    mask[OFF_W3:OFF_B3][w3.ravel()] = False
    mask[OFF_B3 + NOUT:] = False
    m[mask] = b1 * m[mask] + (1 - b1) * g[mask]
    v[mask] = b2 * v[mask] + (1 - b2) * g[mask] ** 2
    mh = m[mask] / (1 - b1 ** step)
    vh = v[mask] / (1 - b2 ** step)
    p[mask] = p[mask] - lr * mh / (np.sqrt(vh) + eps)
    return p, m, v


def features(fields, bounds, mean, inv_std):
    """The closure's 48 features of every interior cell, rows in the order
    (n - ny_start) * nx + (m - nx_start): field f of (u, v, ssh, H, rlh_s)
    at (m + dx, n + dy) is feature 9 f + 3 (dy + 1) + (dx + 1), normalised
    in FP32 as (x - mean) * inv_std and rounded to BF16; 45..47 are zero.
    fields are Fortran-layout arrays over the bounds' array range."""
    b = bounds
    X = np.zeros((b.ny, b.nx, KIN))
    for f in range(5):
        a32 = np.asarray(fields[f]).astype(np.float32)
        z = ((a32 - np.float32(mean[f])) * np.float32(inv_std[f])).astype(np.float32)
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                k = 9 * f + 3 * (dy + 1) + (dx + 1)
                sl = b.sl(b.nx_start + dx, b.nx_end + dx, b.ny_start + dy, b.ny_end + dy)
                X[:, :, k] = bf16(z[sl]).T
    return X.reshape(-1, KIN)
