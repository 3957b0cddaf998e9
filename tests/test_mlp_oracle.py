"""The CPU FP64 oracle of the survival MLP: its backward pass against
central finite differences, and its bf16 rounding against torch's."""
from __future__ import annotations

import numpy as np
import torch

from oracle import mlp_oracle as M


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.standard_normal(20000) * 10.0 ** rng.integers(-6, 6, 20000),
                        [0.0, -0.0, 1.0, 1.00390625, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9]])
    ref = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(M.bf16_round(x), ref)
    bits = torch.tensor(x, dtype=torch.float32).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    assert np.array_equal(M.bf16_bits(x), bits)


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(5)
    p = M.init_params(seed=2)
    B = 24
    X = np.zeros((B, M.IN))
    X[:, :30] = rng.standard_normal((B, 30))
    y = (rng.random(B) < 0.4).astype(np.float64)
    g, _ = M.gradients(p, X, y, emulate=False)
    # parameters from every tensor, avoiding the zero padding columns of W1
    idx = list(rng.choice(np.arange(M.OFF_W1, M.OFF_B1).reshape(M.H, M.IN)[:, :30].ravel(), 8, replace=False))
    for a, b in ((M.OFF_B1, M.OFF_W2), (M.OFF_W2, M.OFF_B2), (M.OFF_B2, M.OFF_W3), (M.OFF_W3, M.OFF_B3),
                 (M.OFF_B3, M.OFF_W4), (M.OFF_W4, M.OFF_B4)):
        idx += list(rng.integers(a, b, 6))
    idx.append(M.OFF_B4)
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (M.loss(pp, X, y) - M.loss(pm, X, y)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(fd), (i, fd, g[i])


def test_emulated_gradient_close_to_exact():
    rng = np.random.default_rng(6)
    p = M.init_params(seed=4)
    X = np.zeros((64, M.IN))
    X[:, :30] = M.bf16_round(rng.standard_normal((64, 30)))
    y = (rng.random(64) < 0.5).astype(np.float64)
    ge, le = M.gradients(p, X, y, emulate=True)
    gx, lx = M.gradients(p, X, y, emulate=False)
    assert np.linalg.norm(ge - gx) / np.linalg.norm(gx) < 0.05
    assert abs(le - lx) < 0.02
