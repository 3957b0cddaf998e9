"""Survival MLP on the GPU (include/bgt_mlp.h) against torch and the CPU
FP64 oracle (oracle/mlp_oracle.py):

* the tcgen05 GEMM against torch's FP32 product of the same bf16 operands
  (tolerance: FP32 accumulation order, 1e-5 relative to the row scale);
* the forward pass against the oracle with bf16 rounding emulated
  (|dp| <= 2e-3: an activation whose FP32 and FP64 values straddle a bf16
  rounding boundary moves by one bf16 ulp);
* the gradients of the hand-written backward kernels against the oracle's
  (relative L2 error <= 1e-2 per tensor, cosine >= 0.9999);
* feature extraction against the same formulas in numpy;
* training on a separable problem.
"""
from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import mlp_oracle as M  # noqa: E402

pytestmark = pytest.mark.gpu


def _bf16(a, dev):
    return torch.tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev).to(torch.bfloat16)


@pytest.mark.parametrize("m,n,k", [(128, 64, 64), (256, 256, 256), (512, 256, 1024), (384, 64, 192),
                                   (1024, 256, 64), (16384, 256, 256), (16384, 256, 4096), (37888, 64, 320),
                                   (32768, 256, 128)])
def test_gemm_matches_torch(m, n, k):
    from bgt import mlp

    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(m * 7 + n + k)
    a = torch.randn(m, k, generator=g).to(dev).to(torch.bfloat16)
    b = torch.randn(n, k, generator=g).to(dev).to(torch.bfloat16)
    c = mlp.gemm_bf16(a, b)
    ref = (a.double() @ b.double().T)
    scale = (a.double().abs() @ b.double().abs().T)
    err = ((c.double() - ref).abs() / scale).max().item()
    assert err < 1e-5, err


def test_gemm_bounded_wait_reports_timeout():
    """The GEMM launched with no MMA issued: every mbarrier wait runs out
    after 1 ms with nothing outstanding, the kernel frees its tensor memory
    and returns, the call reports BGT_ETIMEOUT, and the context stays usable
    (a normal GEMM afterwards is exact)."""
    from bgt import _lib, mlp

    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(5)
    a = torch.randn(256, 128, generator=g).to(dev).to(torch.bfloat16)
    b = torch.randn(64, 128, generator=g).to(dev).to(torch.bfloat16)
    assert mlp.gemm_wait_test(a, b, 1000) == _lib.BGT_ETIMEOUT
    c = mlp.gemm_bf16(a, b)
    ref = a.double() @ b.double().T
    scale = a.double().abs() @ b.double().abs().T
    assert ((c.double() - ref).abs() / scale).max().item() < 1e-5


def _random_net(seed=3, n=1024):
    rng = np.random.default_rng(seed)
    p = M.init_params(seed=seed).astype(np.float32)
    X = np.zeros((n, M.IN))
    X[:, :30] = rng.standard_normal((n, 30))
    X = M.bf16_round(X)
    y = (rng.random(n) < 0.4).astype(np.float32)
    return p, X, y


def test_forward_matches_oracle():
    from bgt import mlp

    dev = torch.device("cuda", 0)
    p, X, _ = _random_net(n=2048)
    net = mlp.SurvivalMLP(max_batch=1024, seed=1)
    net.set_params(p)
    prob = net.forward(_bf16(X, dev)).cpu().numpy()
    ref = M.forward(p, X, emulate=True)["p"]
    assert np.max(np.abs(prob - ref)) < 2e-3
    assert np.mean(np.abs(prob - ref)) < 2e-4


def test_gradients_match_oracle():
    from bgt import mlp

    dev = torch.device("cuda", 0)
    p, X, y = _random_net(seed=4, n=1024)
    net = mlp.SurvivalMLP(max_batch=1024, seed=1)
    net.set_params(p)
    g, loss = net.gradients(_bf16(X, dev), torch.tensor(y, device=dev))
    g = g.cpu().numpy().astype(np.float64)
    gr, lr_ = M.gradients(p, X, y.astype(np.float64), emulate=True)
    assert abs(loss - lr_) < 1e-4
    for a, b in ((M.OFF_W1, M.OFF_B1), (M.OFF_B1, M.OFF_W2), (M.OFF_W2, M.OFF_B2), (M.OFF_B2, M.OFF_W3),
                 (M.OFF_W3, M.OFF_B3), (M.OFF_B3, M.OFF_W4), (M.OFF_W4, M.OFF_B4), (M.OFF_B4, M.N_PARAMS)):
        d, r = g[a:b], gr[a:b]
        rel = np.linalg.norm(d - r) / max(np.linalg.norm(r), 1e-30)
        cos = float(d @ r / (np.linalg.norm(d) * np.linalg.norm(r) + 1e-300))
        assert rel < 1e-2, (a, rel)
        assert cos > 0.9999 or b - a == 1, (a, cos)


def test_features_match_numpy():
    from bgt import mlp

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(9)
    nv, n = 3, 1000
    table = np.zeros((nv, mlp.VARIANT_COLS))
    table[:, :6] = rng.standard_normal((nv, 6)) * 1e-5
    table[:, 6:10] = [0.8, 0.12, 0.0, 0.0]
    table[:, 10:14] = [[11.9, -1.8, 3.7, 0.47]] * nv
    table[:, 14:] = rng.standard_normal((nv, 16))
    var = np.sort(rng.integers(0, nv, n)).astype(np.int32)
    v0 = rng.standard_normal((6, n)) * 1e-3
    v1 = rng.standard_normal((6, n)) * 1e-3
    net = mlp.SurvivalMLP(max_batch=128, seed=1)
    mean = rng.standard_normal(30).astype(np.float32)
    std = (rng.random(30) + 0.5).astype(np.float32)
    net.set_normalization(mean, std)
    x, raw = net.features(torch.tensor(v0, device=dev), torch.tensor(v1, device=dev),
                          torch.tensor(var, device=dev), torch.tensor(table, device=dev), raw=True)
    raw = raw.cpu().numpy()
    T = table[var]
    f = np.zeros((n, 30))
    f[:, 0:6] = v0.T - T[:, :6]
    f[:, 6:22] = T[:, 14:30]
    f[:, 22:28] = v1.T - T[:, :6]
    dp = f[:, 27]
    xb, pxb = f[:, 22] - T[:, 6] * dp, f[:, 23] - T[:, 7] * dp
    yb, pyb = f[:, 24] - T[:, 8] * dp, f[:, 25] - T[:, 9] * dp
    ba, aa, bb, ab = T[:, 10], T[:, 11], T[:, 12], T[:, 13]
    f[:, 28] = np.sqrt(0.5 * ((1 + aa * aa) / ba * xb * xb + 2 * aa * xb * pxb + ba * pxb * pxb))
    f[:, 29] = np.sqrt(0.5 * ((1 + ab * ab) / bb * yb * yb + 2 * ab * yb * pyb + bb * pyb * pyb))
    assert np.allclose(raw, f.astype(np.float32), rtol=1e-6, atol=1e-30)
    xn = x.float().cpu().numpy()
    assert x.shape == (1024, 64) and np.all(xn[:, 30:] == 0) and np.all(xn[n:] == 0)
    exp = M.bf16_round((f.astype(np.float32) - mean) * (np.float32(1) / std))
    assert np.max(np.abs(xn[:n, :30] - exp)) <= 1e-2 * np.max(np.abs(exp))


def test_training_learns_a_separable_rule():
    from bgt import mlp

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(11)
    n = 16384
    X = np.zeros((n, M.IN), np.float32)
    X[:, :30] = rng.standard_normal((n, 30))
    y = ((X[:, 0] ** 2 + X[:, 1] ** 2 + 0.5 * X[:, 2]) > 1.5).astype(np.float32)
    xt = _bf16(X, dev)
    yt = torch.tensor(y, device=dev)
    net = mlp.SurvivalMLP(max_batch=4096, seed=7)
    p0 = net.forward(xt).cpu().numpy()
    l0 = float(np.mean(-(y * np.log(p0 + 1e-12) + (1 - y) * np.log(1 - p0 + 1e-12))))
    hist = net.fit(xt, yt, epochs=8, batch=1024, lr=2e-3, seed=1)
    p = net.forward(xt).cpu().numpy()
    acc = float(np.mean((p > 0.5) == (y > 0.5)))
    assert hist[-1] < 0.5 * l0 and acc > 0.95, (l0, hist, acc)


def test_forward_and_gradients_with_several_tiles_per_cta():
    """The classifier runs its GEMMs on 65,536-row chunks, where each
    persistent CTA drains several 128-row tiles through the double-buffered
    tensor-memory accumulators with the weights held in shared memory: the
    forward pass (bias + ReLU epilogue) on 65,536 rows and the gradients on a
    32,768-sample batch (ReLU-mask epilogue, 74 weight-gradient splits)
    against the oracle, with the single-tile tests' tolerances."""
    from bgt import mlp

    dev = torch.device("cuda", 0)
    p, X, y = _random_net(seed=12, n=65536)
    net = mlp.SurvivalMLP(max_batch=65536, seed=1)
    net.set_params(p)
    prob = net.forward(_bf16(X, dev)).cpu().numpy()
    ref = M.forward(p, X, emulate=True)["p"]
    assert np.max(np.abs(prob - ref)) < 2e-3
    assert np.mean(np.abs(prob - ref)) < 2e-4
    Xb, yb = X[:32768], y[:32768]
    g, loss = net.gradients(_bf16(Xb, dev), torch.tensor(yb, device=dev))
    g = g.cpu().numpy().astype(np.float64)
    gr, lr_ = M.gradients(p, Xb, yb.astype(np.float64), emulate=True)
    assert abs(loss - lr_) < 1e-4
    for a, b in ((M.OFF_W1, M.OFF_B1), (M.OFF_B1, M.OFF_W2), (M.OFF_W2, M.OFF_B2), (M.OFF_B2, M.OFF_W3),
                 (M.OFF_W3, M.OFF_B3), (M.OFF_B3, M.OFF_W4), (M.OFF_W4, M.OFF_B4), (M.OFF_B4, M.N_PARAMS)):
        d, r = g[a:b], gr[a:b]
        rel = np.linalg.norm(d - r) / max(np.linalg.norm(r), 1e-30)
        cos = float(d @ r / (np.linalg.norm(d) * np.linalg.norm(r) + 1e-300))
        assert rel < 1e-2, (a, rel)
        assert cos > 0.9999 or b - a == 1, (a, cos)
