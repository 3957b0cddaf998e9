"""Sharded dynamic-aperture scan across ranks (world size 2, gloo, CPU).

Variants are split into contiguous blocks (bgt.da.shard_range); each rank
scans its block and the per-ray DA radii are all-gathered (bgt.da.
sharded_radii), the one exchange of a sharded scan.  Here the per-rank scan
runs through the oracle; the gathered result must equal the unsharded one
exactly, including an uneven split (3 variants over 2 ranks).
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
        lats = rings.error_variants(N_VAR, seed=3)
        b, e = da.shard_range(N_VAR, rank, world)
        local = _scan(lats[b:e])
        full = da.sharded_radii(local, N_VAR, rank, world)
        q.put((rank, (b, e), full))
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
    full_unsharded = _scan(rings.error_variants(N_VAR, seed=3))
    for _, _, full in res:
        assert full.shape == (N_VAR, 1, GRID["n_angle"])
        assert np.array_equal(full, full_unsharded)
    assert np.any(full_unsharded < GRID["r_max"])  # some rays do lose particles
