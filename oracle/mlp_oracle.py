"""CPU FP64 oracle of the survival MLP -- TEST INFRASTRUCTURE ONLY.

The network has no counterpart in the reference (it prunes the DA scan that
bmad/modules/dynamic_aperture_mod.f90 runs probe by probe), so this oracle is
a plain restatement of the math the device kernels implement
(include/bgt_mlp.h):

    A1 = relu(X W1^T + b1), A2 = relu(A1 W2^T + b2), A3 = relu(A2 W3^T + b3)
    z = A3 w4 + b4, p = sigmoid(z), loss = mean BCE(p, y)

with the flat parameter layout W1[256][64], b1, W2[256][256], b2, W3, b3,
w4[256], b4.  With ``emulate=True`` it rounds to bf16 at the points the
device does (weights, stored activations, stored backward deltas, w4), so the
device's gradients can be checked to the accuracy of FP32 accumulation; with
``emulate=False`` it is the exact FP64 gradient, checked here against finite
differences.  Only tests use this module.
"""
from __future__ import annotations

import numpy as np

IN, H = 64, 256
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * IN
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H * H
OFF_W4 = OFF_B3 + H
OFF_B4 = OFF_W4 + H
N_PARAMS = OFF_B4 + 1


def bf16_round(a) -> np.ndarray:
    """float -> float32 -> bfloat16 (round to nearest even), as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits(a) -> np.ndarray:
    """uint16 bit patterns of bf16_round(a) (for building device inputs)."""
    return (np.ascontiguousarray(bf16_round(a), dtype=np.float32).view(np.uint32) >> 16).astype(np.uint16)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return dict(W1=p[OFF_W1:OFF_B1].reshape(H, IN), b1=p[OFF_B1:OFF_W2], W2=p[OFF_W2:OFF_B2].reshape(H, H),
                b2=p[OFF_B2:OFF_W3], W3=p[OFF_W3:OFF_B3].reshape(H, H), b3=p[OFF_B3:OFF_W4],
                w4=p[OFF_W4:OFF_B4], b4=p[OFF_B4])


def _r(a, emulate):
    return bf16_round(a) if emulate else a


def forward(params, X, emulate: bool = True):
    q = unpack(params)
    W1, W2, W3, w4 = (_r(q[k], emulate) for k in ("W1", "W2", "W3", "w4"))
    X = np.asarray(X, dtype=np.float64)
    A1 = _r(np.maximum(X @ W1.T + q["b1"], 0.0), emulate)
    A2 = _r(np.maximum(A1 @ W2.T + q["b2"], 0.0), emulate)
    A3 = _r(np.maximum(A2 @ W3.T + q["b3"], 0.0), emulate)
    z = A3 @ w4 + q["b4"]
    p = 1.0 / (1.0 + np.exp(-z))
    return dict(X=X, A1=A1, A2=A2, A3=A3, z=z, p=p, W1=W1, W2=W2, W3=W3, w4=w4)


def loss(params, X, y, emulate: bool = False) -> float:
    f = forward(params, X, emulate)
    z = f["z"]
    y = np.asarray(y, dtype=np.float64)
    return float(np.mean(np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z)))))


def gradients(params, X, y, emulate: bool = True):
    """(flat gradient of the mean BCE, loss)."""
    f = forward(params, X, emulate)
    y = np.asarray(y, dtype=np.float64)
    B = X.shape[0]
    g = (f["p"] - y) / B
    dz3 = _r(np.where(f["A3"] > 0, g[:, None] * f["w4"][None, :], 0.0), emulate)
    dz2 = _r(np.where(f["A2"] > 0, dz3 @ f["W3"], 0.0), emulate)
    dz1 = _r(np.where(f["A1"] > 0, dz2 @ f["W2"], 0.0), emulate)
    out = np.zeros(N_PARAMS)
    out[OFF_W1:OFF_B1] = (dz1.T @ f["X"]).ravel()
    out[OFF_B1:OFF_W2] = dz1.sum(axis=0)
    out[OFF_W2:OFF_B2] = (dz2.T @ f["A1"]).ravel()
    out[OFF_B2:OFF_W3] = dz2.sum(axis=0)
    out[OFF_W3:OFF_B3] = (dz3.T @ f["A2"]).ravel()
    out[OFF_B3:OFF_W4] = dz3.sum(axis=0)
    out[OFF_W4:OFF_B4] = f["A3"].T @ g
    out[OFF_B4] = g.sum()
    z = f["z"]
    l = float(np.mean(np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z)))))
    return out, l


def init_params(seed: int = 0, n_features: int = 30) -> np.ndarray:
    """He-uniform weights (padding input columns zero), zero biases."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS)
    w1 = np.zeros((H, IN))
    w1[:, :n_features] = rng.uniform(-1, 1, (H, n_features)) * np.sqrt(6.0 / n_features)
    p[OFF_W1:OFF_B1] = w1.ravel()
    p[OFF_W2:OFF_B2] = rng.uniform(-1, 1, H * H) * np.sqrt(6.0 / H)
    p[OFF_W3:OFF_B3] = rng.uniform(-1, 1, H * H) * np.sqrt(6.0 / H)
    p[OFF_W4:OFF_B4] = rng.uniform(-1, 1, H) * np.sqrt(3.0 / H)
    p[OFF_B1:OFF_W2] = rng.uniform(-0.1, 0.1, H)
    p[OFF_B2:OFF_W3] = rng.uniform(-0.1, 0.1, H)
    p[OFF_B3:OFF_W4] = rng.uniform(-0.1, 0.1, H)
    p[OFF_B4] = 0.05
    return p
