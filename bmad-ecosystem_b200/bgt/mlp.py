"""Survival classifier for dynamic-aperture scans (include/bgt_mlp.h).

A 64-256-256-256-1 MLP (30 features used) with BF16 weights and FP32
accumulation, trained and evaluated on the GPU by the library's own kernels
(tcgen05 tensor-core GEMMs for the hidden layers).  Inputs come from the
tracker itself: the start coordinates, the lattice-error summary of the
particle's variant, and the coordinates and linear actions after the early
turns (:func:`SurvivalMLP.features`).  Device buffers are torch tensors.

No counterpart in the reference: this is the learned pruning step of the
scan driver in :mod:`bgt.learned_da`.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from . import _lib

N_IN = 64
N_FEATURES = 30
HIDDEN = 256
N_PARAMS = 148481
VARIANT_COLS = 30

_mlp_bound = False


def _bind():
    global _mlp_bound
    lib = _lib.load()
    if _mlp_bound:
        return lib
    vp, i32, i64, f32p = C.c_void_p, C.c_int32, C.c_int64, C.POINTER(C.c_float)
    lib.bgt_mlp_create.argtypes = [C.POINTER(vp), i32, C.c_uint64, i32]
    lib.bgt_mlp_destroy.argtypes = [vp]
    lib.bgt_mlp_last_error.argtypes = [vp]
    lib.bgt_mlp_last_error.restype = C.c_char_p
    lib.bgt_mlp_launch_count.argtypes = [vp]
    lib.bgt_mlp_launch_count.restype = i64
    lib.bgt_mlp_get_params.argtypes = [vp, f32p]
    lib.bgt_mlp_set_params.argtypes = [vp, f32p]
    lib.bgt_mlp_forward.argtypes = [vp, vp, i64, vp, vp]
    lib.bgt_mlp_gradients.argtypes = [vp, vp, vp, i32, vp, f32p, vp]
    lib.bgt_mlp_train_step.argtypes = [vp, vp, vp, i32, C.c_float, f32p, vp]
    lib.bgt_mlp_features.argtypes = [vp, vp, i64, i64, vp, vp, i32, vp, vp, vp, vp, vp]
    lib.bgt_mlp_gemm_bf16.argtypes = [vp, i64, vp, i64, i32, i32, i32, vp, vp]
    lib.bgt_mlp_gemm_bf16_wait_test.argtypes = [vp, i64, vp, i64, i32, i32, i32, vp, C.c_uint32, vp]
    _mlp_bound = True
    return lib


def _stream(t):
    import torch

    return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _need(t, dtype, what):
    import torch

    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == dtype and t.is_contiguous()):
        raise ValueError(f"{what} must be a contiguous CUDA tensor of dtype {dtype}")


def gemm_bf16(a, b):
    """C = A . B^T (FP32) with the library's tensor-core GEMM; a [m, k],
    b [n, k] bf16 CUDA tensors (m % 128 == 0, n in {64, 256}, k % 64 == 0)."""
    import torch

    lib = _bind()
    _need(a, torch.bfloat16, "a")
    _need(b, torch.bfloat16, "b")
    m, k = a.shape
    n = b.shape[0]
    c = torch.empty((m, n), dtype=torch.float32, device=a.device)
    rc = lib.bgt_mlp_gemm_bf16(a.data_ptr(), k, b.data_ptr(), b.shape[1], m, n, k, c.data_ptr(), _stream(a))
    if rc != 0:
        raise _lib.BgtError(f"bgt_mlp_gemm_bf16 failed ({rc})")
    return c


def gemm_wait_test(a, b, wait_limit_us: int = 1000) -> int:
    """Return code of the GEMM launched with no MMA issued (its bounded
    mbarrier waits run out after wait_limit_us); BGT_ETIMEOUT expected."""
    import torch

    lib = _bind()
    _need(a, torch.bfloat16, "a")
    _need(b, torch.bfloat16, "b")
    m, k = a.shape
    n = b.shape[0]
    c = torch.empty((m, n), dtype=torch.float32, device=a.device)
    return int(lib.bgt_mlp_gemm_bf16_wait_test(a.data_ptr(), k, b.data_ptr(), b.shape[1], m, n, k, c.data_ptr(),
                                               wait_limit_us, _stream(a)))


def pad_rows(n: int) -> int:
    return -(-n // 128) * 128


class SurvivalMLP:
    def __init__(self, max_batch: int = 65536, seed: int = 1, device: int = 0):
        self.lib = _bind()
        self.device = device
        self.max_batch = max_batch
        h = C.c_void_p()
        rc = self.lib.bgt_mlp_create(C.byref(h), max_batch, seed, device)
        if rc != 0:
            if h:
                self.lib.bgt_mlp_destroy(h)
            raise _lib.BgtError(f"bgt_mlp_create failed ({rc})")
        self.h = h
        import torch

        dev = torch.device("cuda", device)
        self.mean = torch.zeros(N_FEATURES, dtype=torch.float32, device=dev)
        self.inv_std = torch.ones(N_FEATURES, dtype=torch.float32, device=dev)

    def _check(self, rc, what):
        if rc != 0:
            raise _lib.BgtError(f"{what} failed ({rc}): {self.lib.bgt_mlp_last_error(self.h).decode()}")

    @property
    def launch_count(self) -> int:
        return int(self.lib.bgt_mlp_launch_count(self.h))

    # -- parameters --------------------------------------------------------
    def get_params(self) -> np.ndarray:
        p = np.zeros(N_PARAMS, np.float32)
        self._check(self.lib.bgt_mlp_get_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))), "get_params")
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.shape != (N_PARAMS,):
            raise ValueError("parameter vector of the wrong size")
        self._check(self.lib.bgt_mlp_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))), "set_params")

    def set_normalization(self, mean, std):
        import torch

        self.mean = torch.as_tensor(np.asarray(mean, np.float32), device=self.mean.device)
        s = np.asarray(std, np.float64)
        self.inv_std = torch.as_tensor((1.0 / np.where(s > 0, s, 1.0)).astype(np.float32), device=self.mean.device)

    def save(self, path):
        np.savez(path, params=self.get_params(), mean=self.mean.cpu().numpy(), inv_std=self.inv_std.cpu().numpy())

    def load(self, path):
        import torch

        z = np.load(path)
        self.set_params(z["params"])
        self.mean = torch.as_tensor(z["mean"], device=self.mean.device)
        self.inv_std = torch.as_tensor(z["inv_std"], device=self.mean.device)

    # -- network -----------------------------------------------------------
    def forward(self, x):
        """p(lost) for bf16 inputs x [n, 64] (n % 128 == 0)."""
        import torch

        _need(x, torch.bfloat16, "x")
        prob = torch.empty(x.shape[0], dtype=torch.float32, device=x.device)
        self._check(self.lib.bgt_mlp_forward(self.h, x.data_ptr(), x.shape[0], prob.data_ptr(), _stream(x)),
                    "bgt_mlp_forward")
        return prob

    def gradients(self, x, label) -> Tuple["object", float]:
        import torch

        _need(x, torch.bfloat16, "x")
        _need(label, torch.float32, "label")
        g = torch.empty(N_PARAMS, dtype=torch.float32, device=x.device)
        loss = C.c_float()
        self._check(self.lib.bgt_mlp_gradients(self.h, x.data_ptr(), label.data_ptr(), x.shape[0], g.data_ptr(),
                                               C.byref(loss), _stream(x)), "bgt_mlp_gradients")
        return g, float(loss.value)

    def train_step(self, x, label, lr: float, want_loss: bool = False) -> Optional[float]:
        import torch

        _need(x, torch.bfloat16, "x")
        _need(label, torch.float32, "label")
        loss = C.c_float()
        self._check(self.lib.bgt_mlp_train_step(self.h, x.data_ptr(), label.data_ptr(), x.shape[0], lr,
                                                C.byref(loss) if want_loss else None, _stream(x)),
                    "bgt_mlp_train_step")
        return float(loss.value) if want_loss else None

    def fit(self, x, label, epochs: int = 4, batch: int = 8192, lr: float = 2e-3, seed: int = 0,
            verbose: bool = False):
        """Adam on shuffled mini-batches (the tail that does not fill a batch
        is dropped each epoch).  Returns the mean loss of each epoch."""
        import torch

        n = x.shape[0]
        batch = min(batch, self.max_batch, (n // 128) * 128)
        if batch <= 0:
            raise ValueError("not enough samples for one batch of 128")
        g = torch.Generator(device="cpu").manual_seed(seed)
        hist = []
        for ep in range(epochs):
            perm = torch.randperm(n, generator=g).to(x.device)
            losses = []
            for b0 in range(0, n - batch + 1, batch):
                idx = perm[b0:b0 + batch]
                xb = x.index_select(0, idx).contiguous()
                yb = label.index_select(0, idx).contiguous()
                last = b0 + 2 * batch > n
                l = self.train_step(xb, yb, lr, want_loss=last or verbose)
                if l is not None:
                    losses.append(l)
            hist.append(float(np.mean(losses)) if losses else float("nan"))
            if verbose:
                print(f"epoch {ep}: loss {hist[-1]:.5f}", flush=True)
        return hist

    # -- features ----------------------------------------------------------
    def features(self, vec0, vec, variant, table, raw: bool = False, normalized: bool = True):
        """Classifier inputs for particles with start coordinates vec0 and
        current coordinates vec (float64 [6, n] CUDA tensors), variant ids
        (int32 [n]) and the per-variant table (float64 [n_var, 30]).  Returns
        (x bf16 [pad_rows(n), 64] or None, raw float32 [n, 30] or None)."""
        import torch

        _need(vec0, torch.float64, "vec0")
        _need(vec, torch.float64, "vec")
        _need(table, torch.float64, "table")
        if variant is not None:
            _need(variant, torch.int32, "variant")
        n = vec.shape[1]
        dev = vec.device
        x = torch.zeros((pad_rows(n), N_IN), dtype=torch.bfloat16, device=dev) if normalized else None
        r = torch.empty((n, N_FEATURES), dtype=torch.float32, device=dev) if raw else None
        rc = self.lib.bgt_mlp_features(vec0.data_ptr(), vec.data_ptr(), n, vec.shape[1],
                                       variant.data_ptr() if variant is not None else None, table.data_ptr(),
                                       table.shape[0], self.mean.data_ptr(), self.inv_std.data_ptr(),
                                       r.data_ptr() if r is not None else None,
                                       x.data_ptr() if x is not None else None, _stream(vec))
        if rc != 0:
            raise _lib.BgtError(f"bgt_mlp_features failed ({rc})")
        return x, r

    def close(self):
        if getattr(self, "h", None):
            self.lib.bgt_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
