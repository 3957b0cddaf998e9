"""Python call surface of the bgt tracker, shaped after Bmad's multi-particle
tracking routines:

* :meth:`Tracker.track1` / :meth:`Tracker.track_elements` -- ``track1`` and
  ``track_all`` over an element range (``bmad/code/track1.f90:43``,
  ``bmad/code/track_all.f90:25``);
* :meth:`Tracker.track_turns` -- the ``long_term_tracking`` BEAM-mode turn
  loop (``bsim/modules/lt_tracking_mod.f90:1631-1695``) for a whole bunch;
* :meth:`Tracker.track_turns_device` -- the same on device-resident torch
  tensors, enqueued on a CUDA stream;
* :meth:`Tracker.da_scan_grid` -- the dynamic-aperture scan
  (``bmad/modules/dynamic_aperture_mod.f90:27``) on a polar grid.

Particles are held structure-of-arrays in a :class:`Bunch`.  State codes and
loss records follow Bmad (``coord_struct%state``; ``track_state`` = lost-at
element index).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence, Union

import numpy as np

from . import _lib
from . import lattice as L
from . import qp


@dataclass
class Bunch:
    """n particles: vec6[6, n] = (x, px, y, py, z, pz), beta[n], state[n],
    ix_ele_lost[n], ix_turn_lost[n], and optionally the particle times t
    (binary128, an (n, 2) uint64 array: see bgt.qp)."""

    vec6: np.ndarray
    beta: np.ndarray
    state: np.ndarray
    ix_ele_lost: np.ndarray
    ix_turn_lost: np.ndarray
    t: Optional[np.ndarray] = None

    @classmethod
    def from_vec(cls, vec6: np.ndarray, p0c: float, mass: float, with_time: bool = False) -> "Bunch":
        v = np.ascontiguousarray(np.asarray(vec6, dtype=np.float64).reshape(6, -1))
        n = v.shape[1]
        beta = L.beta_of(p0c, v[5], mass)
        t = qp.initial_time(v, beta) if with_time else None
        return cls(v, beta, np.full(n, L.ALIVE, np.int32), np.full(n, -1, np.int32), np.full(n, -1, np.int32), t)

    @property
    def n(self) -> int:
        return self.vec6.shape[1]

    def copy(self) -> "Bunch":
        return Bunch(self.vec6.copy(), self.beta.copy(), self.state.copy(), self.ix_ele_lost.copy(),
                     self.ix_turn_lost.copy(), None if self.t is None else self.t.copy())

    @property
    def time(self) -> np.ndarray:
        """The particle times rounded to double."""
        return qp.to_double(self.t)

    @property
    def n_live(self) -> int:
        return int(np.count_nonzero(self.state == L.ALIVE))


def _check(lib, h, rc, what):
    if rc != 0:
        msg = lib.bgt_last_error(h).decode() if h else ""
        raise _lib.BgtError(f"{what} failed ({rc}): {msg}")


class Tracker:
    """Device element tables for one ring and any number of variants of it
    (same element sequence, per-variant values).  absolute_time sets
    bmad_com%absolute_time_tracking: the RF phase from the particle time,
    which every bunch then carries."""

    def __init__(self, lattices: Union[L.Lattice, Sequence[L.Lattice]], device: int = 0,
                 tuning: Optional[dict] = None, absolute_time: bool = False, absolute_time_ref_shift: bool = True):
        lats: List[L.Lattice] = [lattices] if isinstance(lattices, L.Lattice) else list(lattices)
        if not lats:
            raise ValueError("no lattice")
        n_ele = len(lats[0])
        for lat in lats:
            if len(lat) != n_ele:
                raise ValueError("all variants must have the same number of elements")
        self.lib = _lib.load()
        self.lattice = lats[0]
        self.n_ele = n_ele
        self.n_variants = len(lats)
        arr = (_lib.BgtElement * (n_ele * len(lats)))()
        seen = {}
        for v, lat in enumerate(lats):
            for i, e in enumerate(lat.elements):
                k = _lib.element_key(e)
                c = seen.get(k)
                if c is None:
                    c = seen[k] = _lib.to_bgt_element(e)
                arr[v * n_ele + i] = c
        sp = _lib.BgtSpecies(lats[0].species.mass, lats[0].species.charge, 1, 1e3, 1 if absolute_time else 0,
                             1 if absolute_time_ref_shift else 0)
        self.absolute_time = bool(absolute_time)
        self.species = lats[0].species
        self.p0c = lats[0].p0c
        h = C.c_void_p()
        rc = self.lib.bgt_create(C.byref(h), arr, n_ele, len(lats), C.byref(sp), device)
        if rc != 0:
            raise _lib.BgtError(f"bgt_create failed ({rc}): {self.lib.bgt_last_error(None).decode()}")
        self.h = h
        self.device = device
        if tuning:
            self.set_tuning(**tuning)

    # -- tuning -----------------------------------------------------------
    def set_tuning(self, threads_per_block=0, blocks_per_sm=0, turns_per_launch=0, compact_every=0, table_mode=0,
                   wait_limit_us=0, test_skip_table_copy=0):
        t = _lib.BgtTuning(threads_per_block, blocks_per_sm, turns_per_launch, compact_every, table_mode,
                           wait_limit_us, test_skip_table_copy)
        _check(self.lib, self.h, self.lib.bgt_set_tuning(self.h, C.byref(t)), "bgt_set_tuning")

    def get_tuning(self) -> dict:
        t = _lib.BgtTuning()
        _check(self.lib, self.h, self.lib.bgt_get_tuning(self.h, C.byref(t)), "bgt_get_tuning")
        return {k: getattr(t, k) for k, _ in _lib.BgtTuning._fields_}

    def table_bytes(self) -> int:
        b = C.c_int64()
        n = C.c_int32()
        _check(self.lib, self.h, self.lib.bgt_table_info(self.h, C.byref(b), C.byref(n)), "bgt_table_info")
        return b.value

    @property
    def launch_count(self) -> int:
        return int(self.lib.bgt_kernel_launch_count(self.h))

    # -- tracking ---------------------------------------------------------
    def make_bunch(self, vec6, with_time: Optional[bool] = None) -> Bunch:
        """A bunch at the ring start; with_time (default: with absolute time
        tracking) gives it init_coord's particle times."""
        wt = self.absolute_time if with_time is None else with_time
        return Bunch.from_vec(vec6, self.p0c, self.species.mass, with_time=wt)

    @staticmethod
    def _t_ptr(b: Bunch):
        if b.t is None:
            return None
        if b.t.shape != (b.n, 2) or b.t.dtype != np.uint64 or not b.t.flags["C_CONTIGUOUS"]:
            raise ValueError("bunch.t must be a C-contiguous (n, 2) uint64 array of binary128 times")
        return b.t.ctypes.data

    def track_turns(self, bunch: Bunch, n_turns: int, turn0: int = 0,
                    variant: Optional[np.ndarray] = None) -> Bunch:
        """Track the bunch in place for n_turns turns (host buffers)."""
        b = bunch
        var = None
        if variant is not None:
            var = np.ascontiguousarray(variant, dtype=np.int32)
            if var.shape != (b.n,):
                raise ValueError("variant must have one entry per particle")
        rc = self.lib.bgt_track_turns(self.h, _lib.ptr(b.vec6, C.c_double), _lib.ptr(b.beta, C.c_double),
                                      self._t_ptr(b), _lib.ptr(b.state, C.c_int32),
                                      _lib.ptr(b.ix_ele_lost, C.c_int32),
                                      _lib.ptr(b.ix_turn_lost, C.c_int32),
                                      _lib.ptr(var, C.c_int32) if var is not None else None, b.n, turn0, n_turns)
        _check(self.lib, self.h, rc, "bgt_track_turns")
        return b

    def track_elements(self, bunch: Bunch, e_begin: int, e_end: int,
                       variant: Optional[np.ndarray] = None) -> Bunch:
        """track_all over table elements [e_begin, e_end) (0-based positions)."""
        b = bunch
        var = None if variant is None else np.ascontiguousarray(variant, dtype=np.int32)
        rc = self.lib.bgt_track_elements(self.h, _lib.ptr(b.vec6, C.c_double), _lib.ptr(b.beta, C.c_double),
                                         self._t_ptr(b), _lib.ptr(b.state, C.c_int32),
                                         _lib.ptr(b.ix_ele_lost, C.c_int32),
                                         _lib.ptr(var, C.c_int32) if var is not None else None, b.n, e_begin,
                                         e_end)
        _check(self.lib, self.h, rc, "bgt_track_elements")
        return b

    def track1(self, bunch: Bunch, position: int, variant=None) -> Bunch:
        """track1 through the element at 0-based table position `position`."""
        return self.track_elements(bunch, position, position + 1, variant)

    def track_turns_device(self, vec6, beta, state, ix_ele_lost, ix_turn_lost, n_turns: int, turn0: int = 0,
                           stream=None, variant=None, t=None):
        """Track device-resident torch tensors in place, enqueued on `stream`
        (a torch.cuda.Stream; default: the current stream).  `variant` (int32
        CUDA tensor, sorted) selects each particle's lattice variant; with
        more than one variant the call synchronises the stream once.  `t`
        (a contiguous (n, 2) int64 CUDA tensor of binary128 bits) carries the
        particle times."""
        import torch

        if stream is None:
            stream = torch.cuda.current_stream(vec6.device)
        checks = [(vec6, torch.float64), (beta, torch.float64), (state, torch.int32), (ix_ele_lost, torch.int32),
                  (ix_turn_lost, torch.int32)]
        if variant is not None:
            checks.append((variant, torch.int32))
        for x, dt in checks:
            if not x.is_cuda or x.dtype != dt or not x.is_contiguous():
                raise ValueError("device tensors must be contiguous CUDA tensors of the documented dtype")
        n = beta.numel()
        if vec6.numel() != 6 * n or (variant is not None and variant.numel() != n):
            raise ValueError("vec6 must hold 6*n values and variant n")
        if t is not None and (not t.is_cuda or t.dtype != torch.int64 or not t.is_contiguous() or t.numel() != 2 * n):
            raise ValueError("t must be a contiguous (n, 2) int64 CUDA tensor of binary128 bits")
        rc = self.lib.bgt_track_turns_device(self.h, vec6.data_ptr(), beta.data_ptr(),
                                             t.data_ptr() if t is not None else None, state.data_ptr(),
                                             ix_ele_lost.data_ptr(), ix_turn_lost.data_ptr(),
                                             variant.data_ptr() if variant is not None else None, n, turn0,
                                             n_turns, C.c_void_p(stream.cuda_stream))
        _check(self.lib, self.h, rc, "bgt_track_turns_device")

    def device_status(self, stream=None):
        """Wait for `stream` (default: the current stream) and raise BgtError
        if a device-buffer call since the last check hit a table-staging
        timeout on the device (the flag is cleared)."""
        import torch

        if stream is None:
            stream = torch.cuda.current_stream(torch.device("cuda", self.device))
        rc = self.lib.bgt_device_status(self.h, C.c_void_p(stream.cuda_stream))
        _check(self.lib, self.h, rc, "bgt_device_status")

    def da_scan_grid(self, ref_orbit: np.ndarray, n_angle: int, angle_min: float, angle_max: float,
                     n_radius: int, r_max: float, y_scale: float, n_turns: int, n_variants: Optional[int] = None,
                     return_survival: bool = False):
        """Polar-grid DA scan.  ref_orbit[v, d, 6] is the starting reference
        orbit of variant v at momentum setting d.  Returns da_radius[v, d, a]
        (and survive_turns[v, d, a, r] if asked)."""
        ref = np.ascontiguousarray(ref_orbit, dtype=np.float64)
        nv = ref.shape[0] if n_variants is None else n_variants
        nd = ref.shape[1]
        out = np.zeros((nv, nd, n_angle), dtype=np.float64)
        surv = np.zeros((nv, nd, n_angle, n_radius), dtype=np.int32) if return_survival else None
        rc = self.lib.bgt_da_scan_grid(self.h, _lib.ptr(ref, C.c_double), nv, nd, n_angle, angle_min, angle_max,
                                       n_radius, r_max, y_scale, n_turns, _lib.ptr(out, C.c_double),
                                       _lib.ptr(surv, C.c_int32) if surv is not None else None)
        _check(self.lib, self.h, rc, "bgt_da_scan_grid")
        return (out, surv) if return_survival else out

    def close(self):
        if getattr(self, "h", None):
            self.lib.bgt_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fp64_peak_tflops(device: int = 0) -> float:
    lib = _lib.load()
    out = C.c_double()
    rc = lib.bgt_fp64_peak_tflops(device, C.byref(out))
    if rc != 0:
        raise _lib.BgtError(f"bgt_fp64_peak_tflops failed ({rc})")
    return out.value
