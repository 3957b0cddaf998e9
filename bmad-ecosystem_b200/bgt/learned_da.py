"""Classifier-pruned dynamic-aperture scans.

The plain scan (:func:`bgt.da.plain_scan`) tracks every polar-grid probe of
every variant for the full turn count.  Here every probe is tracked for the
first `early` turns (64); a survival classifier (:class:`bgt.mlp.SurvivalMLP`)
then reads the start coordinates, the variant's lattice-error summary, and
the coordinates and linear actions at turn `early`, and gives p(lost).
Probes still alive at that turn are

* retired as lost when p > p_hi (0.98) -- the only early retirement the
  method allows: "only particles it marks confidently as lost are retired
  early";
* tracked to the full turn count by the FP64 tracker otherwise: every probe
  of the uncertainty band p <= p_hi, every probe within `boundary_cells`
  grid cells of the predicted DA boundary of its ray, and a random audit
  fraction (2 %) of the rest.

`p_lo` > 0 (default 0) also retires confident survivors (p < p_lo) as
surviving without tracking them: a faster scan outside that rule, kept as a
measured comparison only.

The DA radius of each ray then comes from the tracked outcomes where they
exist and the classifier's labels elsewhere, and the audit measures the
classifier's error rate on probes it would have retired.  Training data come
from the tracker itself: a staged plain scan (snapshot at turn `early`,
outcome at the full turn count) of the training variants, optionally with
extra probes jittered inside each grid cell.

No counterpart in the reference; the grid, the reference orbits and the DA
radius rule are those of :mod:`bgt.da` (dynamic_aperture_mod.f90).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import da
from . import lattice as L
from .mlp import SurvivalMLP, pad_rows


@dataclass
class ScanProblem:
    tracker: object
    lattices: Sequence[L.Lattice]
    optics: da.VariantOptics
    ref: np.ndarray  # [v, d, 6]
    deltas: Sequence[float]
    n_angle: int
    angle_min: float
    angle_max: float
    n_radius: int
    r_max: float
    yscale: float
    n_turns: int
    summary: np.ndarray  # [v, 16]
    table: np.ndarray = field(default=None)  # [v, 30]

    def __post_init__(self):
        if self.table is None:
            self.table = np.concatenate([self.optics.table(), self.summary], axis=1)

    @property
    def n_variants(self):
        return self.ref.shape[0]

    @property
    def per_variant(self):
        return len(self.deltas) * self.n_angle * self.n_radius

    def grid(self, n_turns: Optional[int] = None) -> dict:
        return dict(n_angle=self.n_angle, angle_min=self.angle_min, angle_max=self.angle_max,
                    n_radius=self.n_radius, r_max=self.r_max, yscale=self.yscale,
                    n_turns=self.n_turns if n_turns is None else n_turns)


def setup(tracker, lattices, grid, k2_nominal=None, yscale: Optional[float] = None) -> ScanProblem:
    """Per-variant optics through the GPU one-turn map, reference orbits at
    the grid's momentum offsets, and the error summaries."""
    opt = da.variant_optics(da.tracker_one_turn(tracker), len(lattices))
    ref = da.reference_orbits(opt, grid.deltas)
    ys = yscale if yscale is not None else da.y_scale(float(np.mean(opt.beta_a)), float(np.mean(opt.beta_b)))
    return ScanProblem(tracker, lattices, opt, ref, tuple(grid.deltas), grid.n_angle, grid.angle_min,
                       grid.angle_max, grid.n_radius, grid.r_max, ys, grid.n_turns,
                       da.error_summary(lattices, k2_nominal))


def _device():
    import torch

    return torch.device("cuda", torch.cuda.current_device())


def grid_probes(pb: ScanProblem, v_begin: int, v_end: int, jitter_seed: Optional[int] = None):
    """Start coordinates (float64 [6, n] CUDA) and variant ids of the grid
    probes of variants [v_begin, v_end), in (variant, delta, angle, radius)
    order.  With jitter_seed, each probe moves uniformly inside its grid
    cell (+-half a radius step and +-half an angle step; training data)."""
    import torch

    ref = pb.ref[v_begin:v_end]
    if jitter_seed is None:
        v6 = da.grid_initial_conditions(ref, pb.n_angle, pb.angle_min, pb.angle_max, pb.n_radius, pb.r_max,
                                        pb.yscale)
    else:
        rng = np.random.default_rng(jitter_seed)
        nv, nd = ref.shape[:2]
        ang = da.ray_angles(pb.n_angle, pb.angle_min, pb.angle_max)
        rad = da.grid_radii(pb.n_radius, pb.r_max)
        dth = (ang[1] - ang[0]) if pb.n_angle > 1 else 0.0
        dr = rad[1] - rad[0]
        shape = (nv, nd, pb.n_angle, pb.n_radius)
        a = ang[None, None, :, None] + (rng.random(shape) - 0.5) * dth
        r = np.maximum(rad[None, None, None, :] + (rng.random(shape) - 0.5) * dr, 0.0)
        v = np.repeat(ref[:, :, None, None, :], pb.n_angle, axis=2).repeat(pb.n_radius, axis=3).copy()
        v[..., 0] += np.cos(a) * r
        v[..., 2] += np.sin(a) * r * pb.yscale
        v6 = np.ascontiguousarray(v.reshape(-1, 6).T)
    dev = _device()
    var = np.repeat(np.arange(v_begin, v_end, dtype=np.int32), pb.per_variant)
    return torch.tensor(v6, device=dev).contiguous(), torch.tensor(var, device=dev)


def tracking_order(pb: ScanProblem, nv: int):
    """Probe index held by each tracking position: radius-major inside each
    (variant, delta), so a warp tracks one radius across the angles and the
    warps of a CTA are lost at similar turns (no idling at the end-of-tile
    barrier).  Results do not depend on the order."""
    import torch

    idx = np.arange(nv * pb.per_variant).reshape(nv, len(pb.deltas), pb.n_angle, pb.n_radius)
    return torch.tensor(idx.transpose(0, 1, 3, 2).ravel(), device=_device())


class _Bunch:
    """Device particle arrays of a scan, held in tracking order
    (`order[k]` = probe index at tracking position k)."""

    def __init__(self, vec6, variant, p0c, mass, order=None):
        import torch

        self.order = order
        if order is not None:
            vec6 = vec6[:, order]
            variant = variant[order]
        self.vec = vec6.contiguous().clone()
        self.var = variant.contiguous()
        n = vec6.shape[1]
        # beta as the one-launch scan computes it: pc / sqrt(pc^2 + m^2)
        pc = (1 + vec6[5]) * p0c
        self.beta = (pc / torch.sqrt(pc * pc + mass * mass)).contiguous()
        self.state = torch.ones(n, dtype=torch.int32, device=vec6.device)
        self.ixe = torch.full((n,), -1, dtype=torch.int32, device=vec6.device)
        self.ixt = torch.full((n,), -1, dtype=torch.int32, device=vec6.device)

    def probe_order(self, t):
        """A tracking-order array (last axis) in probe order."""
        import torch

        if self.order is None:
            return t
        out = torch.empty_like(t)
        out[..., self.order] = t
        return out

    def subset(self, idx):
        b = _Bunch.__new__(_Bunch)
        b.order = None
        b.vec = self.vec[:, idx].contiguous()
        b.beta = self.beta[idx].contiguous()
        b.state = self.state[idx].contiguous()
        b.ixe = self.ixe[idx].contiguous()
        b.ixt = self.ixt[idx].contiguous()
        b.var = self.var[idx].contiguous()
        return b

    def track(self, tracker, n_turns, turn0):
        if n_turns > 0:
            tracker.track_turns_device(self.vec, self.beta, self.state, self.ixe, self.ixt, n_turns, turn0=turn0,
                                       variant=self.var)


def survive_turns(state, ixt, n_turns):
    import torch

    return torch.where(state == 1, torch.full_like(ixt, n_turns), ixt)


@dataclass
class StagedScan:
    vec0: object  # [6, n] start coordinates
    vec_early: object  # [6, n] at turn `early`
    variant: object
    alive_early: object  # bool [n]
    survive: object  # int32 [n] turns survived (n_turns = all)
    early: int
    n_turns: int
    wall_s: float
    particle_turns: int


def staged_scan(pb: ScanProblem, v_begin: int, v_end: int, early: int = 64, n_turns: Optional[int] = None,
                jitter_seed: Optional[int] = None) -> StagedScan:
    """Plain scan of variants [v_begin, v_end) in two launches: `early`
    turns, a snapshot, then the rest.  Bit-identical to the one-launch scan."""
    import torch

    nt = pb.n_turns if n_turns is None else n_turns
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    vec0, var = grid_probes(pb, v_begin, v_end, jitter_seed)
    tr = pb.tracker
    b = _Bunch(vec0, var, tr.p0c, tr.species.mass, tracking_order(pb, v_end - v_begin))
    b.track(tr, early, 0)
    snap = b.probe_order(b.vec)
    alive = b.probe_order(b.state) == 1
    b.track(tr, nt - early, early)
    surv = b.probe_order(survive_turns(b.state, b.ixt, nt))
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    pt = int(torch.clamp(surv, max=nt).sum().item())
    return StagedScan(vec0, snap, var, alive, surv, early, nt, wall, pt)


def compacted_scan(pb: ScanProblem, v_begin: int, v_end: int, early: int = 64, n_turns: Optional[int] = None,
                   retune_subset: bool = True) -> da.DAResult:
    """Plain scan of variants [v_begin, v_end) in two launches and no
    classifier: every probe `early` turns, then only the probes still alive,
    packed densely in tracking order (variants stay sorted), to the full
    turn count.  On the error rings ~70 % of the probes are lost within the
    first turns; in a one-launch scan their lanes stay in the tiles of the
    long-lived probes, here the second launch holds live probes only.  Each
    probe's arithmetic does not depend on its lane, so the outcomes equal
    the one-launch scan's bit for bit.  With `retune_subset` the second
    launch's shape is re-tuned on the packed set (a few 2-turn trial
    launches) and the tracker's tuning restored afterwards."""
    import torch

    nt = pb.n_turns if n_turns is None else n_turns
    nv = v_end - v_begin
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    vec0, var = grid_probes(pb, v_begin, v_end)
    tr = pb.tracker
    b = _Bunch(vec0, var, tr.p0c, tr.species.mass, tracking_order(pb, nv))
    b.track(tr, early, 0)
    idx = torch.nonzero(b.state == 1).view(-1)  # tracking positions, ascending
    if idx.numel() and nt > early:
        sub = b.subset(idx)
        saved = tr.get_tuning()
        try:
            if retune_subset:
                from . import autotune

                autotune.tune(tr, sub.vec.cpu().numpy(), turns=2, sample=int(idx.numel()),
                              variant=sub.var.cpu().numpy())
            sub.track(tr, nt - early, early)
        finally:
            tr.set_tuning(**saved)
        b.state[idx] = sub.state
        b.ixt[idx] = sub.ixt
        b.ixe[idx] = sub.ixe
        b.vec[:, idx] = sub.vec
    surv = b.probe_order(survive_turns(b.state, b.ixt, nt))
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    s = surv.cpu().numpy().astype(np.int32)
    radius = radius_of(pb, s >= nt, nv)
    pt = int(np.minimum(s, nt).sum())
    return da.DAResult(radius, s.reshape(nv, len(pb.deltas), pb.n_angle, pb.n_radius),
                       da.ray_angles(pb.n_angle, pb.angle_min, pb.angle_max), da.grid_radii(pb.n_radius, pb.r_max),
                       nt, wall, pt)


def radius_of(pb: ScanProblem, survive_label, nv: int) -> np.ndarray:
    """DA radius per ray from a boolean survive label per probe."""
    s = np.asarray(survive_label).reshape(nv, len(pb.deltas), pb.n_angle, pb.n_radius)
    return da.radius_from_survival(np.where(s, 1, 0), 1, pb.r_max)


def training_set(pb: ScanProblem, scans: Sequence[StagedScan], net: SurvivalMLP):
    """Raw features and labels (1 = lost before the full turn count) of the
    probes alive at turn `early`, concatenated over staged scans."""
    import torch

    table = torch.tensor(pb.table, device=_device())
    raws, labels = [], []
    for s in scans:
        _, raw = net.features(s.vec0, s.vec_early, s.variant, table, raw=True, normalized=False)
        m = s.alive_early
        raws.append(raw[m])
        labels.append((s.survive[m] < s.n_turns).float())
    return torch.cat(raws), torch.cat(labels)


def gather_rows(t, group=None):
    """Concatenate a [n_rank, ...] tensor over all ranks in rank order (rows
    per rank may differ): the training samples of a scan sharded by variant,
    so that every rank trains the same network on all of them."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return t
    world = dist.get_world_size(group)
    n = torch.tensor([t.shape[0]], dtype=torch.int64, device=t.device)
    ns = [torch.empty_like(n) for _ in range(world)]
    dist.all_gather(ns, n, group=group)
    ns = [int(x.item()) for x in ns]
    buf = torch.zeros((max(ns),) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
    buf[:t.shape[0]] = t
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return torch.cat([p[:k] for p, k in zip(parts, ns)])


def normalized_inputs(net: SurvivalMLP, raw):
    """bf16 [pad_rows(n), 64] network inputs from raw features (n, 30)."""
    import torch

    n = raw.shape[0]
    x = torch.zeros((pad_rows(n), 64), dtype=torch.float32, device=raw.device)
    x[:n, :30] = (raw - net.mean) * net.inv_std
    return x.to(torch.bfloat16)


def train(net: SurvivalMLP, raw, label, epochs: int = 6, batch: int = 8192, lr: float = 2e-3, seed: int = 0,
          set_normalization: bool = True, verbose: bool = False):
    """Set the input normalisation from the training features (unless
    fine-tuning) and train; returns (per-epoch loss, wall seconds)."""
    import torch

    if set_normalization:
        mean = raw.double().mean(0).float().cpu().numpy()
        std = raw.double().std(0).float().cpu().numpy()
        net.set_normalization(mean, np.where(std > 0, std, 1.0))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    n = (raw.shape[0] // 128) * 128  # whole batches of 128
    x = normalized_inputs(net, raw[:n])
    hist = net.fit(x, label[:n].float().contiguous(), epochs=epochs, batch=batch, lr=lr, seed=seed,
                   verbose=verbose)
    torch.cuda.synchronize()
    return hist, time.perf_counter() - t0


@dataclass
class PrunedResult:
    radius: np.ndarray  # [v, d, a]
    survive_label: np.ndarray  # bool [n]
    tracked: np.ndarray  # bool [n] tracked to the full turn count
    p_lost: np.ndarray  # float [n] (NaN for probes lost before turn `early`)
    wall_s: float
    particle_turns: int
    n_probes: int
    n_tracked: int
    n_retired_lost: int
    n_retired_survive: int
    audit_n: int
    audit_errors: int


def pruned_scan(pb: ScanProblem, net: SurvivalMLP, v_begin: int, v_end: int, early: int = 64,
                n_turns: Optional[int] = None, p_hi: float = 0.98, p_lo: float = 0.0, audit: float = 0.02,
                boundary_cells: int = 2, seed: int = 0, retune_subset: bool = True) -> PrunedResult:
    """The kept probes are far fewer than the grid, so their tracking is
    bound by one particle's turn latency rather than by throughput; with
    `retune_subset` the launch shape for them is re-tuned on the kept set
    itself (a few 2-turn trial launches) and the scan's tuning restored
    afterwards."""
    import torch

    nt = pb.n_turns if n_turns is None else n_turns
    nv = v_end - v_begin
    nd, na, nr = len(pb.deltas), pb.n_angle, pb.n_radius
    dev = _device()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    vec0, var = grid_probes(pb, v_begin, v_end)
    tr = pb.tracker
    b = _Bunch(vec0, var, tr.p0c, tr.species.mass, tracking_order(pb, nv))
    b.track(tr, early, 0)
    alive = b.probe_order(b.state) == 1
    table = torch.tensor(pb.table, device=dev)
    x, _ = net.features(vec0, b.probe_order(b.vec).contiguous(), var, table)
    n = vec0.shape[1]
    p = net.forward(x)[:n]
    # predicted DA boundary of each ray: the first probe lost or predicted lost
    pred_lost = torch.where(alive, p > 0.5, torch.ones_like(alive))
    g = pred_lost.view(nv, nd, na, nr)
    any_lost = g.any(dim=-1)
    first = torch.where(any_lost, g.int().argmax(dim=-1), torch.full_like(any_lost, nr, dtype=torch.int64))
    r_idx = torch.arange(nr, device=dev).view(1, 1, 1, nr)
    near = ((r_idx - first.unsqueeze(-1)).abs() <= boundary_cells).view(-1)
    band = (p >= p_lo) & (p <= p_hi)  # p_lo = 0: every probe not confidently lost
    gen = torch.Generator(device="cpu").manual_seed(seed)
    aud = (torch.rand(n, generator=gen) < audit).to(dev)
    track_mask = alive & (band | near | aud)
    # tracking positions of the kept probes, ascending: variants stay sorted
    idx = torch.nonzero(track_mask[b.order]).view(-1)
    m = int(idx.numel())
    label = torch.where(alive, p <= 0.5, torch.zeros_like(alive))
    actual = label.clone()
    tracked_turns = 0
    if m:
        sub = b.subset(idx)
        saved = tr.get_tuning()
        try:
            if retune_subset:
                from . import autotune

                autotune.tune(tr, sub.vec.cpu().numpy(), turns=2, sample=m, variant=sub.var.cpu().numpy())
            sub.track(tr, nt - early, early)
        finally:
            tr.set_tuning(**saved)
        actual[b.order[idx]] = sub.state == 1
        tracked_turns = int((survive_turns(sub.state, sub.ixt, nt) - early).clamp(min=0).sum().item())
    early_turns = int(torch.clamp(survive_turns(b.state, b.ixt, early), max=early).sum().item())
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    lab = actual.cpu().numpy()
    radius = radius_of(pb, lab, nv)
    al = alive.cpu().numpy()
    bandn = band.cpu().numpy()
    tm = track_mask.cpu().numpy()
    aud_c = aud.cpu().numpy() & al & ~bandn
    pred = label.cpu().numpy()
    pn = np.where(al, p.cpu().numpy(), np.nan)
    return PrunedResult(radius, lab, tm, pn, wall, early_turns + tracked_turns, n, m,
                        int(np.sum(al & ~tm & (pn > p_hi))), int(np.sum(al & ~tm & (pn < p_lo))),
                        int(aud_c.sum()), int(np.sum(aud_c & (pred != lab))))


def ranking_mismatches(da_a: np.ndarray, da_b: np.ndarray) -> dict:
    """Compare two rankings of the same variants by mean DA radius: pairwise
    order disagreements (Kendall distance), Spearman rho and the number of
    variants whose rank position differs."""
    a = np.argsort(np.argsort(-da_a, kind="stable"), kind="stable")
    b = np.argsort(np.argsort(-da_b, kind="stable"), kind="stable")
    n = len(a)
    disc = 0
    for i in range(n):
        disc += int(np.sum(np.sign(a[i] - a[i + 1:]) != np.sign(b[i] - b[i + 1:])))
    rho = 1 - 6 * float(np.sum((a - b) ** 2)) / (n * (n * n - 1)) if n > 1 else 1.0
    return {"pairs": n * (n - 1) // 2, "discordant_pairs": disc, "spearman": rho,
            "rank_position_mismatches": int(np.sum(a != b))}
