"""Launch-shape autotuner for the tracking kernel.

Candidates are the (particles per CTA, resident CTAs per SM) pairs the library
is compiled for -- i.e. register caps of 128/96/80/64 per thread traded
against occupancy --, for some of them the element table read from global
memory instead of shared memory (frees shared memory for more resident CTAs
when tables are large), and, for lossy workloads, the compaction interval.  Each
candidate tracks a sample of the real bunch for a few turns on the device
(CUDA events on the launching stream); the fastest per particle.turn wins.
Results are cached per (table bytes, lattice name, particle count) in memory
and, when a path is given, in a JSON file.
"""
from __future__ import annotations

import json
import os
from pathlib import Path
from typing import Dict, Iterable, Optional, Tuple

import numpy as np

from . import _lib

SHAPES: Tuple[Tuple[int, int], ...] = ((64, 8), (64, 10), (64, 12), (64, 16), (128, 4), (128, 5), (128, 6),
                                       (128, 8), (256, 2), (256, 3), (256, 4))

# shapes compiled with the element table read from global memory (table_mode 2 and 3)
GLOBAL_TABLE_SHAPES: Tuple[Tuple[int, int], ...] = ((128, 3), (128, 4), (128, 5), (256, 2), (256, 3))

_cache: Dict[str, dict] = {}


def _key(tracker, n: int, lossy: bool) -> str:
    return f"{tracker.lattice.name}:{tracker.table_bytes()}:{tracker.n_variants}:{n}:{int(lossy)}"


def candidates(shapes: Iterable[Tuple[int, int]] = SHAPES, compact_options: Iterable[int] = (0,)) -> list:
    """The tunings tried: every compiled shape with each compaction
    interval, and, for the shapes also compiled for global-memory tables,
    the table in shared memory (0) or in global memory with CTA tiles (2)
    or warp tiles (3); shapes compiled only for global-memory tables last."""
    shapes = list(shapes)
    compact_options = list(compact_options)
    out = [dict(threads_per_block=tpb, blocks_per_sm=bps, compact_every=ce, turns_per_launch=0, table_mode=tm)
           for (tpb, bps) in shapes for ce in compact_options
           for tm in ((0, 2, 3) if (tpb, bps) in GLOBAL_TABLE_SHAPES else (0,))]
    out += [dict(threads_per_block=tpb, blocks_per_sm=bps, compact_every=0, turns_per_launch=0, table_mode=tm)
            for (tpb, bps) in GLOBAL_TABLE_SHAPES if (tpb, bps) not in shapes for tm in (2, 3)]
    return out


def _cuda_timer(tracker, vec6: np.ndarray, pick: np.ndarray, variant: Optional[np.ndarray], turns: int):
    """A function timing the tracker's current tuning on the sample
    vec6[:, pick] (CUDA events on the launching stream, best of two)."""
    import torch

    m = len(pick)
    dev = torch.device("cuda", tracker.device)
    base = torch.tensor(np.ascontiguousarray(vec6[:, pick]), dtype=torch.float64, device=dev)
    var_t = (torch.tensor(np.ascontiguousarray(variant[pick], dtype=np.int32), device=dev)
             if variant is not None else None)
    pz = base[5]
    pc = (1 + pz) * tracker.p0c
    beta0 = pc / torch.sqrt(pc * pc + tracker.species.mass ** 2)
    stream = torch.cuda.current_stream(dev)
    return lambda: _time_shape(tracker, base, beta0, var_t, m, turns, stream, dev)


def _time_shape(tracker, base, beta0, var_t, m, turns, stream, dev) -> float:
    import torch

    best = None
    for rep in range(2):  # first repetition warms up
        v = base.clone()
        b = beta0.clone()
        st = torch.ones(m, dtype=torch.int32, device=dev)
        ie = torch.full((m,), -1, dtype=torch.int32, device=dev)
        it = torch.full((m,), -1, dtype=torch.int32, device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        tracker.track_turns_device(v, b, st, ie, it, turns, stream=stream, variant=var_t)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    return best


def tune(tracker, vec6: np.ndarray, turns: int = 4, shapes: Iterable[Tuple[int, int]] = SHAPES,
         compact_options: Iterable[int] = (0,), sample: int = 200_000, cache_file: Optional[str] = None,
         verbose: bool = False, variant: Optional[np.ndarray] = None, timer=None) -> dict:
    """Pick the fastest tuning for tracking `vec6` (6, n) with `tracker`;
    sets it on the tracker and returns it.  `variant` (sorted int32 [n])
    assigns the particles to lattice variants; the sample is then spread
    evenly over the bunch so that every variant's share is represented.
    `timer` (no arguments, milliseconds of the tracker's current tuning)
    replaces the CUDA timing of the sample."""
    n = vec6.shape[1]
    lossy = any(c > 0 for c in compact_options)
    key = _key(tracker, n, lossy)
    if cache_file and not _cache and os.path.exists(cache_file):
        try:
            _cache.update(json.loads(Path(cache_file).read_text()))
        except (OSError, ValueError):
            pass
    if key in _cache:
        tracker.set_tuning(**_cache[key]["tuning"])
        return _cache[key]["tuning"]

    m = min(n, sample)
    pick = np.linspace(0, n - 1, m).astype(np.int64) if variant is not None else np.arange(m)
    if timer is None:
        timer = _cuda_timer(tracker, vec6, pick, variant, turns)
    results = []
    for tun in candidates(shapes, compact_options):
        tracker.set_tuning(**tun)
        try:
            best = timer()
        except _lib.BgtError:
            continue  # shape not available for this table (e.g. table larger than shared memory)
        results.append((best, tun))
        if verbose:
            print(f"  tune {tun}: {best:.3f} ms")
    if not results:
        raise _lib.BgtError("no launch shape can run this table")
    results.sort(key=lambda r: r[0])
    choice = results[0][1]
    tracker.set_tuning(**choice)
    _cache[key] = {"tuning": choice, "ms": results[0][0], "turns": turns, "sample": m,
                   "all": [(ms, t) for ms, t in results]}
    if cache_file:
        try:
            Path(cache_file).write_text(json.dumps(_cache, indent=1))
        except OSError:
            pass
    return choice


def last_results(tracker, n: int, lossy: bool = False) -> Optional[dict]:
    return _cache.get(_key(tracker, n, lossy))
