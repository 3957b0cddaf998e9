"""The C ABI as a multi-threaded caller and a failing device see it.

* Re-entrancy: the reference calls track1 from OpenMP threads
  (bmad/multiparticle/beam_utils.f90:69-74) and track_many from the parallel
  sections of its DA scan (bmad/modules/dynamic_aperture_mod.f90:163-196), so
  the hook installed there (bgt_track_elements) is called by many threads on
  one handle at once.  Eight threads calling it concurrently must get exactly
  what the same calls made one after the other get.
* Bounded waits: a kernel whose element-table copy never lands gives up after
  the tuning's wait limit, reports BGT_ETIMEOUT (host-buffer calls) or sets
  the handle's device status (device-buffer calls), and leaves the context
  usable.  The test arms the copy's barrier without issuing the copy
  (tuning.test_skip_table_copy), so nothing is in flight when the wait runs
  out.
"""
import ctypes as C
import threading

import numpy as np
import pytest

from bgt import _lib
from bgt import lattice as L
from bgt import rings
from bgt.track import Tracker

from helpers import random_particles, zoo_lattice

pytestmark = pytest.mark.gpu

N_THREADS = 8


def _calls(lat):
    """Per thread: a bunch and the element ranges it tracks through, in
    order (track_all over consecutive ranges, then whole passes)."""
    n_ele = len(lat)
    out = []
    for k in range(N_THREADS):
        v0 = random_particles(600 + 97 * k, seed=300 + k, scale=1.5)
        cuts = sorted(set([0, n_ele] + [int(x) for x in np.linspace(0, n_ele, 4 + k % 3)[1:-1]]))
        ranges = list(zip(cuts[:-1], cuts[1:])) + [(0, n_ele)] * 3
        out.append((v0, ranges))
    return out


def _run(tr, v0, ranges):
    b = tr.make_bunch(v0.copy())
    for e0, e1 in ranges:
        tr.track_elements(b, e0, e1)
    return b


def test_concurrent_track_elements_equal_serial():
    lat = zoo_lattice()
    tr = Tracker(lat)
    work = _calls(lat)
    serial = [_run(tr, v0, r) for v0, r in work]
    results = [None] * N_THREADS
    errors = []
    start = threading.Barrier(N_THREADS)

    def worker(k):
        try:
            start.wait()
            for _ in range(3):  # several rounds so that calls overlap
                results[k] = _run(tr, *work[k])
        except Exception as e:  # reported below, with the thread
            errors.append((k, repr(e)))

    th = [threading.Thread(target=worker, args=(k,)) for k in range(N_THREADS)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors, errors
    for k in range(N_THREADS):
        a, b = results[k], serial[k]
        assert np.array_equal(a.state, b.state), k
        assert np.array_equal(a.ix_ele_lost, b.ix_ele_lost), k
        assert np.array_equal(a.vec6, b.vec6), k
        assert np.array_equal(a.beta, b.beta), k
    assert any((b.state != L.ALIVE).any() for b in serial)  # losses on the way


def test_concurrent_turns_and_device_calls_on_one_handle():
    """Host-buffer turn loops on four threads and device-buffer calls on two
    private streams, all on one handle at once, equal the serial calls."""
    import torch

    lat = rings.fodo_ring(apertures=True)
    tr = Tracker(lat)
    beams = [rings.gaussian_beam(rings.BeamSpec(1500 + 300 * k, 4e-6, 2e-6, 3e-3, 2e-3, seed=400 + k))
             for k in range(6)]
    ref = []
    for k, v0 in enumerate(beams):
        b = tr.make_bunch(v0.copy())
        tr.track_turns(b, 12, turn0=k)
        ref.append(b)
    out = [None] * 6
    errors = []
    start = threading.Barrier(6)

    def host(k):
        try:
            start.wait()
            b = tr.make_bunch(beams[k].copy())
            tr.track_turns(b, 12, turn0=k)
            out[k] = (b.vec6, b.state, b.ix_ele_lost, b.ix_turn_lost)
        except Exception as e:
            errors.append((k, repr(e)))

    def device(k):
        try:
            v0 = beams[k]
            n = v0.shape[1]
            s = torch.cuda.Stream()
            with torch.cuda.stream(s):
                dv = torch.tensor(v0, dtype=torch.float64, device="cuda").contiguous()
                db = torch.tensor(L.beta_of(lat.p0c, v0[5], lat.species.mass), device="cuda")
                ds = torch.ones(n, dtype=torch.int32, device="cuda")
                de = torch.full((n,), -1, dtype=torch.int32, device="cuda")
                dt = torch.full((n,), -1, dtype=torch.int32, device="cuda")
            start.wait()
            tr.track_turns_device(dv, db, ds, de, dt, 12, turn0=k, stream=s)
            tr.device_status(s)
            out[k] = (dv.cpu().numpy(), ds.cpu().numpy(), de.cpu().numpy(), dt.cpu().numpy())
        except Exception as e:
            errors.append((k, repr(e)))

    th = [threading.Thread(target=host if k < 4 else device, args=(k,)) for k in range(6)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors, errors
    for k in range(6):
        v, s, e, t = out[k]
        assert np.array_equal(v, ref[k].vec6), k
        assert np.array_equal(s, ref[k].state), k
        assert np.array_equal(e, ref[k].ix_ele_lost), k
        assert np.array_equal(t, ref[k].ix_turn_lost), k


def test_staging_wait_runs_out_and_the_handle_recovers():
    import torch

    lat = rings.fodo_ring(apertures=True)
    tr = Tracker(lat)
    v0 = rings.gaussian_beam(rings.BeamSpec(2000, 4e-6, 2e-6, 3e-3, 2e-3, seed=501))
    good = tr.make_bunch(v0.copy())
    tr.track_turns(good, 5)
    # host-buffer call: BGT_ETIMEOUT, the caller's arrays left as they were
    tr.set_tuning(wait_limit_us=20000, test_skip_table_copy=1)
    b = tr.make_bunch(v0.copy())
    with pytest.raises(_lib.BgtError, match=r"\(-5\)"):
        tr.track_turns(b, 5)
    assert np.array_equal(b.vec6, v0)
    # device-buffer call: returns at once, the failure shows in the status
    n = v0.shape[1]
    dv = torch.tensor(v0, dtype=torch.float64, device="cuda").contiguous()
    db = torch.tensor(L.beta_of(lat.p0c, v0[5], lat.species.mass), device="cuda")
    ds = torch.ones(n, dtype=torch.int32, device="cuda")
    de = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    dt = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    tr.track_turns_device(dv, db, ds, de, dt, 5)
    with pytest.raises(_lib.BgtError, match=r"\(-5\)"):
        tr.device_status()
    tr.device_status()  # the check cleared the flag
    # the same handle and the same context work normally afterwards
    tr.set_tuning()
    b = tr.make_bunch(v0.copy())
    tr.track_turns(b, 5)
    assert np.array_equal(b.vec6, good.vec6) and np.array_equal(b.state, good.state)
    tr.track_turns_device(dv, db, ds, de, dt, 5)
    tr.device_status()
    assert np.array_equal(dv.cpu().numpy(), good.vec6)
    assert np.array_equal(de.cpu().numpy(), good.ix_ele_lost)
