"""Sharded dynamic-aperture scan across ranks (world size 2, gloo, CPU).

The code path bench.py's DA workloads take under torchrun: variants are
split into contiguous blocks (bgt.da.shard_range), each rank scans its block
through bgt.da.sharded_scan, which all-gathers the per-ray DA radii
(bgt.da.sharded_radii, the one exchange of a sharded scan) and reduces wall
time (max) and particle.turns (sum); the classifier's training rows are
all-gathered with bgt.learned_da.gather_rows so every rank trains on all of
them.  Here the per-rank scan runs through the oracle (no GPU); the gathered
result must equal the unsharded one exactly, including an uneven split
(3 variants over 2 ranks) and uneven row counts.
"""
from __future__ import annotations

import datetime
import math
import multiprocessing as mp
import os
import socket
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]

GRID = dict(n_angle=3, angle_min=0.0, angle_max=math.pi, n_radius=6, r_max=0.03, yscale=0.6)
N_TURNS = 12
N_VAR = 3


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _scan(lats):
    from bgt import da
    from helpers import oracle_da_survival

    ref = np.zeros((len(lats), 1, 6))
    surv = oracle_da_survival(lats, ref, n_turns=N_TURNS, **GRID)
    return da.radius_from_survival(surv, N_TURNS, GRID["r_max"])


def _scan_result(lats):
    """The per-rank scan as a DAResult, the shape bgt.da.plain_scan returns."""
    import time

    from bgt import da
    from helpers import oracle_da_survival

    t0 = time.perf_counter()
    ref = np.zeros((len(lats), 1, 6))
    surv = oracle_da_survival(lats, ref, n_turns=N_TURNS, **GRID)
    radius = da.radius_from_survival(surv, N_TURNS, GRID["r_max"])
    return da.DAResult(radius, surv, da.ray_angles(GRID["n_angle"]), da.grid_radii(GRID["n_radius"], GRID["r_max"]),
                       N_TURNS, time.perf_counter() - t0, int(np.minimum(surv, N_TURNS).sum()))


def _worker(rank, world, port, q):
    sys.path.insert(0, str(ROOT / "bmad-ecosystem_b200"))
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist

    from bgt import da, rings

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        import torch

        from bgt import learned_da as LD

        lats = rings.error_variants(N_VAR, seed=3)
        sh = da.sharded_scan(lambda b, e: _scan_result(lats[b:e]), N_VAR, rank, world)
        # training rows: rank r holds 3 + 2r rows of 4 features valued by rank
        rows = torch.full((3 + 2 * rank, 4), float(rank))
        g = LD.gather_rows(rows)
        q.put((rank, (sh.begin, sh.end), sh.radius, sh.particle_turns, sh.local.particle_turns, sh.wall_s,
               sh.local.wall_s, g.numpy()))
    finally:
        dist.destroy_process_group()


def test_shard_range_covers_all():
    from bgt import da

    for n in (1, 3, 7, 256):
        for w in (1, 2, 3, 8):
            got = []
            for r in range(w):
                b, e = da.shard_range(n, r, w)
                got.extend(range(b, e))
            assert got == list(range(n))


def test_sharded_scan_equals_unsharded(oracle_lib):
    from bgt import rings

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    ranges = sorted(r[1] for r in res)
    assert ranges == [(0, 2), (2, 3)]
    full_unsharded = _scan_result(rings.error_variants(N_VAR, seed=3))
    total_pt = sum(r[4] for r in res)
    max_wall = max(r[6] for r in res)
    expect_rows = np.concatenate([np.zeros((3, 4)), np.ones((5, 4))])
    for _, _, full, pt, _, wall, _, rows in res:
        assert full.shape == (N_VAR, 1, GRID["n_angle"])
        assert np.array_equal(full, full_unsharded.radius)
        assert pt == total_pt == full_unsharded.particle_turns
        assert wall == max_wall
        assert np.array_equal(rows, expect_rows)
    assert np.any(full_unsharded.radius < GRID["r_max"])  # some rays do lose particles
