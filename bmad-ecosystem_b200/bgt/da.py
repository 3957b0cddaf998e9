"""Dynamic-aperture scans on the GPU tracker.

Restates the setup of ``dynamic_aperture_scan``
(bmad/modules/dynamic_aperture_mod.f90:27-207):

* ray angles ``angle_j = j * (max - min) / (n - 1) + min``, one angle -> the
  midpoint (:88-95);
* the reference orbit of each momentum setting: with the RF on, the 6D closed
  orbit at the start plus ``pz * (eta_x, etap_x, eta_y, etap_y, 0, 1)``
  (:132-136);

and replaces the amplitude bisection of ``dynamic_aperture_point`` (:335-388)
by a polar grid: radii ``r_k = k * r_max / (n_radius - 1)`` along each ray,
``(x, y) = ref + (r cos a, r sin a * y_scale)``, every point tracked for the
full turn count in one launch.  The DA radius of a ray is the largest grid
radius below the first lost point (the lower bracket ``x0`` of the bisection).

Variants: every function takes per-variant arrays; the tracker holds all
variants' element tables and runs them in one launch.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass
from typing import Callable, Optional, Sequence

import numpy as np

from . import lattice as L

# one turn of a batch: (vec6[6, m], variant[m]) -> vec6 after one turn
BatchOneTurn = Callable[[np.ndarray, np.ndarray], np.ndarray]


def ray_angles(n_angle: int, angle_min: float = 0.0, angle_max: float = math.pi) -> np.ndarray:
    """dynamic_aperture_mod.f90:88-95."""
    if n_angle == 1:
        return np.array([(angle_min + angle_max) / 2])
    da = (angle_max - angle_min) / (n_angle - 1)
    return np.array([j * da + angle_min for j in range(n_angle)])


def grid_radii(n_radius: int, r_max: float) -> np.ndarray:
    dr = r_max / (n_radius - 1)
    return np.array([k * dr for k in range(n_radius)])


@dataclass
class VariantOptics:
    """Per-variant linear optics at the start of the ring."""
    closed_orbit: np.ndarray  # [v, 6]
    eta: np.ndarray  # [v, 4]  (eta_x, etap_x, eta_y, etap_y)
    beta_a: np.ndarray
    alpha_a: np.ndarray
    beta_b: np.ndarray
    alpha_b: np.ndarray
    tune_a: np.ndarray
    tune_b: np.ndarray

    @property
    def n_variants(self) -> int:
        return self.closed_orbit.shape[0]

    def table(self) -> np.ndarray:
        """[v, 14]: closed orbit (6), eta (4), beta_a, alpha_a, beta_b, alpha_b."""
        return np.concatenate([self.closed_orbit, self.eta, self.beta_a[:, None], self.alpha_a[:, None],
                               self.beta_b[:, None], self.alpha_b[:, None]], axis=1)


def tracker_one_turn(tracker) -> BatchOneTurn:
    """One-turn map of every variant through the GPU tracker (host buffers)."""

    def f(vec6: np.ndarray, variant: np.ndarray) -> np.ndarray:
        b = tracker.make_bunch(np.ascontiguousarray(vec6, dtype=np.float64))
        tracker.track_turns(b, 1, variant=variant)
        if np.any(b.state != 1):
            raise RuntimeError("particle lost while probing the one-turn map")
        return b.vec6

    return f


def _twiss_plane(m2: np.ndarray):
    c = 0.5 * (m2[0, 0] + m2[1, 1])
    if abs(c) >= 1:
        raise ValueError("unstable plane (|cos mu| >= 1)")
    mu = math.acos(c)
    if m2[0, 1] < 0:
        mu = 2 * math.pi - mu
    s = math.sin(mu)
    return m2[0, 1] / s, (m2[0, 0] - m2[1, 1]) / (2 * s), mu / (2 * math.pi)


def variant_optics(one_turn: BatchOneTurn, n_variants: int, h_newton: float = 1e-8, h_matrix: float = 1e-6,
                   tol: float = 1e-13, max_iter: int = 20) -> VariantOptics:
    """6D closed orbit (Newton, all variants at once), the 6x6 one-turn
    matrix by central differences, Twiss of the transverse 2x2 blocks and the
    periodic dispersion (I - M4) eta = M[0:4, 5]."""
    nv = n_variants
    co = np.zeros((nv, 6))
    var7 = np.repeat(np.arange(nv, dtype=np.int32), 7)
    for _ in range(max_iter):
        pts = np.repeat(co[:, :, None], 7, axis=2)  # [v, 6, 7]
        for k in range(6):
            pts[:, k, 1 + k] += h_newton
        flat = np.ascontiguousarray(pts.transpose(1, 0, 2).reshape(6, nv * 7))
        out = one_turn(flat, var7).reshape(6, nv, 7).transpose(1, 0, 2)
        f0 = out[:, :, 0] - pts[:, :, 0]
        jac = (out[:, :, 1:] - out[:, :, :1]) / h_newton  # [v, 6, 6]
        step = np.linalg.solve(jac - np.eye(6)[None], -f0[:, :, None])[:, :, 0]
        co = co + step
        if np.max(np.abs(step)) < tol:
            break
    var12 = np.repeat(np.arange(nv, dtype=np.int32), 12)
    pts = np.repeat(co[:, :, None], 12, axis=2)
    for k in range(6):
        pts[:, k, 2 * k] += h_matrix
        pts[:, k, 2 * k + 1] -= h_matrix
    flat = np.ascontiguousarray(pts.transpose(1, 0, 2).reshape(6, nv * 12))
    out = one_turn(flat, var12).reshape(6, nv, 12).transpose(1, 0, 2)
    m = (out[:, :, 0::2] - out[:, :, 1::2]) / (2 * h_matrix)  # [v, 6, 6]
    ba, aa, qa, bb, ab, qb = (np.zeros(nv) for _ in range(6))
    eta = np.zeros((nv, 4))
    for v in range(nv):
        ba[v], aa[v], qa[v] = _twiss_plane(m[v, 0:2, 0:2])
        bb[v], ab[v], qb[v] = _twiss_plane(m[v, 2:4, 2:4])
        eta[v] = np.linalg.solve(np.eye(4) - m[v, 0:4, 0:4], m[v, 0:4, 5])
    return VariantOptics(co, eta, ba, aa, bb, ab, qa, qb)


def reference_orbits(optics: VariantOptics, deltas: Sequence[float]) -> np.ndarray:
    """ref[v, d, 6] = closed orbit + pz * (eta_x, etap_x, eta_y, etap_y, 0, 1),
    dynamic_aperture_mod.f90:132-136 (RF on)."""
    nv = optics.n_variants
    ref = np.zeros((nv, len(deltas), 6))
    for d, pz in enumerate(deltas):
        ref[:, d, :] = optics.closed_orbit
        ref[:, d, 0:4] += pz * optics.eta
        ref[:, d, 5] += pz
    return ref


def y_scale(beta_a: float, beta_b: float) -> float:
    """Vertical grid scale sqrt(beta_y / beta_x) at the start."""
    return math.sqrt(beta_b / beta_a)


def grid_initial_conditions(ref: np.ndarray, n_angle: int, angle_min: float, angle_max: float, n_radius: int,
                            r_max: float, yscale: float) -> np.ndarray:
    """vec6[6, n] in (variant, delta, angle, radius) order, the same starting
    points the one-launch scan builds on the device."""
    nv, nd = ref.shape[:2]
    ang = ray_angles(n_angle, angle_min, angle_max)
    cs = np.array([[math.cos(a), math.sin(a)] for a in ang])  # host C library, like the device scan
    rad = grid_radii(n_radius, r_max)
    v6 = np.repeat(ref[:, :, None, None, :], n_angle, axis=2).repeat(n_radius, axis=3).copy()
    v6[..., 0] = v6[..., 0] + cs[None, None, :, None, 0] * rad[None, None, None, :]
    v6[..., 2] = v6[..., 2] + (cs[None, None, :, None, 1] * rad[None, None, None, :]) * yscale
    return np.ascontiguousarray(v6.reshape(-1, 6).T)


def radius_from_survival(survive: np.ndarray, n_turns: int, r_max: float) -> np.ndarray:
    """survive[..., r] (turns survived) -> DA radius per ray: the largest grid
    radius below the first point that did not survive n_turns."""
    n_radius = survive.shape[-1]
    dr = r_max / (n_radius - 1)
    lost = survive < n_turns
    first = np.where(lost.any(axis=-1), lost.argmax(axis=-1), n_radius)
    return np.where(first > 0, dr * (first - 1), 0.0)


@dataclass
class DAResult:
    radius: np.ndarray  # [v, d, a] (m)
    survive_turns: Optional[np.ndarray]  # [v, d, a, r]
    angles: np.ndarray
    radii: np.ndarray
    n_turns: int
    wall_s: float
    particle_turns: int = 0


def plain_scan(tracker, ref: np.ndarray, n_angle: int, angle_min: float, angle_max: float, n_radius: int,
               r_max: float, yscale: float, n_turns: int, return_survival: bool = True) -> DAResult:
    """Every grid point of every variant tracked n_turns turns in one launch
    (bgt_da_scan_grid)."""
    t0 = time.perf_counter()
    res = tracker.da_scan_grid(ref, n_angle, angle_min, angle_max, n_radius, r_max, yscale, n_turns,
                               n_variants=ref.shape[0], return_survival=return_survival)
    wall = time.perf_counter() - t0
    radius, surv = (res if return_survival else (res, None))
    pt = int(np.minimum(surv, n_turns).sum()) if surv is not None else 0
    return DAResult(radius, surv, ray_angles(n_angle, angle_min, angle_max), grid_radii(n_radius, r_max), n_turns,
                    wall, pt)


def da_error(radius: np.ndarray, radius_ref: np.ndarray) -> float:
    """Relative DA-radius error: sum |r - r_ref| / sum r_ref over all rays."""
    den = float(np.sum(radius_ref))
    return float(np.sum(np.abs(radius - radius_ref))) / den if den > 0 else 0.0


def error_summary(lattices: Sequence[L.Lattice], k2_nominal: Optional[Sequence[float]] = None) -> np.ndarray:
    """[v, 16] lattice-error summary of each variant, in units of the error
    sigmas: rms x/y offset and roll of the quadrupoles (3) and of the
    sextupoles (3), rms a_n and b_n for n = 3..6 over both families (8), and
    the relative SF/SD k2 deviation from nominal (2)."""
    out = np.zeros((len(lattices), 16))
    for v, lat in enumerate(lattices):
        cols = []
        for key in ("quadrupole", "sextupole"):
            es = [e for e in lat.elements if e.key == key]
            for name, sig in (("x_offset", 50e-6), ("y_offset", 50e-6), ("tilt", 100e-6)):
                vals = np.array([e.values.get(name, 0.0) for e in es])
                cols.append(math.sqrt(float(np.mean(vals * vals))) / sig if len(vals) else 0.0)
        es = [e for e in lat.elements if e.key in ("quadrupole", "sextupole")]
        for arr in ("a_pole", "b_pole"):
            for n in range(3, 7):
                vals = np.array([getattr(e, arr).get(n, 0.0) for e in es])
                cols.append(math.sqrt(float(np.mean(vals * vals))) / 1e-4 if len(vals) else 0.0)
        k2 = [None, None]
        for e in lat.elements:
            if e.key == "sextupole":
                k = e.values.get("k2", 0.0)
                if k > 0 and k2[0] is None:
                    k2[0] = k
                if k < 0 and k2[1] is None:
                    k2[1] = k
        for j in range(2):
            nom = k2_nominal[j] if k2_nominal is not None else None
            cols.append((k2[j] / nom - 1) / 0.3 if (nom and k2[j] is not None) else 0.0)
        out[v] = cols
    return out


def shard_range(n: int, rank: int, world: int):
    """Contiguous block [begin, end) of n items for `rank` of `world`."""
    per = -(-n // world)
    b = min(n, rank * per)
    return b, min(n, b + per)


def sharded_radii(local: np.ndarray, n_variants: int, rank: int, world: int, group=None) -> np.ndarray:
    """Gather per-variant DA radii [v_local, d, a] from every rank into the
    full [n_variants, d, a] array (torch.distributed all_gather; the one
    exchange of a sharded scan).  Each rank holds shard_range(n_variants)."""
    import torch
    import torch.distributed as dist

    per = -(-n_variants // world)
    shape = local.shape[1:]
    buf = np.zeros((per,) + shape)
    buf[:local.shape[0]] = local
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    t = torch.from_numpy(buf).to(dev)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    full = np.concatenate([p.cpu().numpy() for p in parts], axis=0)
    return full[:n_variants]


@dataclass
class ShardedScan:
    radius: np.ndarray  # [n_variants, d, a], all variants (gathered)
    local: DAResult  # this rank's scan of its block
    begin: int  # this rank's block of variants [begin, end)
    end: int
    wall_s: float  # max over ranks
    particle_turns: int  # summed over ranks


def sharded_scan(scan, n_variants: int, rank: int = 0, world: int = 1, group=None) -> ShardedScan:
    """A DA scan sharded by lattice variant: `scan(v_begin, v_end)` -> DAResult
    runs on this rank's contiguous block (shard_range), then the per-ray radii
    of every variant are all-gathered (sharded_radii) -- the scan's one
    exchange; wall time is the max over ranks, particle.turns the sum.  The
    reference's analogue is the angle-parallel OpenMP scan
    (bmad/modules/dynamic_aperture_mod.f90:182-196)."""
    b, e = shard_range(n_variants, rank, world)
    res = scan(b, e)
    if world == 1:
        return ShardedScan(res.radius, res, b, e, res.wall_s, res.particle_turns)
    import torch
    import torch.distributed as dist

    full = sharded_radii(res.radius, n_variants, rank, world, group)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    w = torch.tensor([res.wall_s], dtype=torch.float64, device=dev)
    dist.all_reduce(w, op=dist.ReduceOp.MAX, group=group)
    pt = torch.tensor([float(res.particle_turns)], dtype=torch.float64, device=dev)
    dist.all_reduce(pt, op=dist.ReduceOp.SUM, group=group)
    return ShardedScan(full, res, b, e, float(w.item()), int(pt.item()))
