"""The allocation-free entry point (bgt_track_turns_device_noalloc) against
the regular device entry point, through the C ABI.

Some callers cannot let the library allocate device memory -- a host whose
framework owns the GPU's memory through its own caching allocator, or a loop
that must not allocate per call.  The allocation-free entry point keeps its
element table and scratch counters in a fixed device array inside the
library instead.  Two calls in a row (different lattices and particles) must
reproduce the regular entry point's results; both use the same kernel and
table contents, so the comparison is exact (tolerance 0).  This file is named
so pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from bgt import _lib
from bgt import lattice as L
from bgt import rings
from bgt.track import Tracker

pytestmark = pytest.mark.gpu


def _device_arrays(torch, v0, lat):
    n = v0.shape[1]
    return (torch.tensor(v0, dtype=torch.float64, device="cuda").contiguous(),
            torch.tensor(L.beta_of(lat.p0c, v0[5], lat.species.mass), device="cuda"),
            torch.ones(n, dtype=torch.int32, device="cuda"),
            torch.full((n,), -1, dtype=torch.int32, device="cuda"),
            torch.full((n,), -1, dtype=torch.int32, device="cuda"))


def _noalloc(torch, lat, arrays, turns, tuning=None):
    lib = _lib.load()
    els = (_lib.BgtElement * len(lat.elements))(*[_lib.to_bgt_element(e) for e in lat.elements])
    sp = _lib.BgtSpecies(lat.species.mass, lat.species.charge, 1, 1e3)
    v, b, s, ie, it = arrays
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream()
    status = torch.full((1,), 7, dtype=torch.int32, device="cuda")
    tun = None if tuning is None else C.byref(_lib.BgtTuning(*tuning))
    rc = lib.bgt_track_turns_device_noalloc(els, len(lat.elements), C.byref(sp), v.data_ptr(), b.data_ptr(),
                                            s.data_ptr(), ie.data_ptr(), it.data_ptr(), b.numel(), 0, turns, tun,
                                            0, C.c_void_p(stream.cuda_stream), status.data_ptr(), err, 256)
    assert rc == 0, err.value.decode()
    torch.cuda.synchronize()
    assert int(status.item()) == 0  # no table-staging wait ran out


def _regular(torch, lat, arrays, turns, tuning=None):
    tr = Tracker(lat)
    if tuning is not None:
        tr.set_tuning(*tuning)
    tr.track_turns_device(*arrays, turns)
    torch.cuda.synchronize()
    tr.device_status()


def _large_table_lattice():
    """The ring with every quadrupole and sextupole carrying its own offsets,
    roll and multipole errors, and every drift and bend a length of its own:
    ~209 KB of distinct records, more than the kernel's shared memory holds
    next to its per-particle state (224 KB less 26 KB of quadrupole memos at
    128 threads), less than the allocation-free scratch array."""
    lat = rings.error_variants(1, seed=17)[0]
    for i, e in enumerate(lat.elements):
        if e.key in ("drift", "sbend"):
            e.values["l"] = e.values["l"] * (1 + 1e-9 * i)
    return lat


@pytest.mark.parametrize("dummy", [0])
def test_noalloc_matches_regular_entry_point_twice(dummy):
    torch = pytest.importorskip("torch")
    cases = [
        (rings.fodo_ring(apertures=True), rings.BeamSpec(3000, 4e-6, 2e-6, 3e-3, 2e-3, seed=91), 25, None),
        (rings.error_variants(1, seed=9)[0], rings.BeamSpec(2000, 1e-6, 5e-7, 3e-3, 1e-3, seed=92), 10, None),
        # (256, 2) with compaction every 3 turns and launches of 4 turns
        (rings.fodo_ring(apertures=True), rings.BeamSpec(2500, 4e-6, 2e-6, 3e-3, 2e-3, seed=93), 11,
         (256, 2, 4, 3, 0)),
    ]
    for lat, spec, turns, tun in cases:  # calls in a row through the same scratch array
        v0 = rings.gaussian_beam(spec)
        a = _device_arrays(torch, v0, lat)
        _noalloc(torch, lat, a, turns, tun)
        r = _device_arrays(torch, v0, lat)
        _regular(torch, lat, r, turns, tun)
        for x, y in zip(a, r):
            assert torch.equal(x, y)


def test_noalloc_table_read_in_place_matches_regular():
    """A table between the shared-memory budget and the scratch array's
    size is read from the array in place; results equal the regular entry
    point's."""
    torch = pytest.importorskip("torch")
    lat = _large_table_lattice()
    tb = Tracker(lat).table_bytes()
    assert (224 - 26) * 1024 < tb < 256 * 1024 - 256, tb
    v0 = rings.gaussian_beam(rings.BeamSpec(1500, 1e-6, 5e-7, 3e-3, 1e-3, seed=94))
    for _ in range(2):
        a = _device_arrays(torch, v0, lat)
        _noalloc(torch, lat, a, 4)
        r = _device_arrays(torch, v0, lat)
        _regular(torch, lat, r, 4)
        for x, y in zip(a, r):
            assert torch.equal(x, y)


def test_noalloc_rejects_oversized_table():
    torch = pytest.importorskip("torch")
    lat = rings.fodo_ring()
    # distinct elements defeat the record sharing
    for i, e in enumerate(lat.elements):
        if e.key == "drift":
            e.values["l"] = 0.3 + 1e-9 * i
            e.key = "quadrupole"
            e.values["k1"] = 0.01 + 1e-6 * i
            e.fringe_type = "none"
    for _ in range(4):  # ~3600 elements, ~2900 distinct records: > 256 KiB
        lat.elements += [x.copy() for x in lat.elements[:700]]
    for i, e in enumerate(lat.elements):
        e.ix_ele = i + 1
        if e.key == "quadrupole":
            e.values["k1"] = 0.01 + 1e-7 * i
    lib = _lib.load()
    els = (_lib.BgtElement * len(lat.elements))(*[_lib.to_bgt_element(e) for e in lat.elements])
    sp = _lib.BgtSpecies(lat.species.mass, lat.species.charge, 1, 1e3)
    v = torch.zeros(6, dtype=torch.float64, device="cuda")
    b = torch.ones(1, dtype=torch.float64, device="cuda")
    s = torch.ones(1, dtype=torch.int32, device="cuda")
    ie = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    err = C.create_string_buffer(256)
    rc = lib.bgt_track_turns_device_noalloc(els, len(lat.elements), C.byref(sp), v.data_ptr(), b.data_ptr(),
                                            s.data_ptr(), ie.data_ptr(), None, 1, 0, 1, None, 0, None, None, err,
                                            256)
    assert rc == _lib.BGT_ETOOLARGE, (rc, err.value)
    assert b"scratch array holds" in err.value
    # a launch shape outside (128, 4) / (256, 2) is refused before anything runs
    small = rings.fodo_ring()
    els = (_lib.BgtElement * len(small.elements))(*[_lib.to_bgt_element(e) for e in small.elements])
    bad = _lib.BgtTuning(64, 8, 0, 0, 0)
    rc = lib.bgt_track_turns_device_noalloc(els, len(small.elements), C.byref(sp), v.data_ptr(), b.data_ptr(),
                                            s.data_ptr(), ie.data_ptr(), None, 1, 0, 1, C.byref(bad), 0, None, None,
                                            err, 256)
    assert rc == _lib.BGT_EINVAL and b"tuning" in err.value


def test_noalloc_reports_a_staging_timeout_then_recovers():
    """A call whose table-staging wait runs out writes 1 to d_status and
    leaves the particles untouched; the next call clears the flag and tracks
    normally."""
    torch = pytest.importorskip("torch")
    lat = rings.fodo_ring(apertures=True)
    v0 = rings.gaussian_beam(rings.BeamSpec(1200, 4e-6, 2e-6, 3e-3, 2e-3, seed=95))
    lib = _lib.load()
    els = (_lib.BgtElement * len(lat.elements))(*[_lib.to_bgt_element(e) for e in lat.elements])
    sp = _lib.BgtSpecies(lat.species.mass, lat.species.charge, 1, 1e3)
    a = _device_arrays(torch, v0, lat)
    v, b, s, ie, it = a
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    err = C.create_string_buffer(256)
    skip = _lib.BgtTuning(128, 4, 0, 0, 0, 20000, 1)
    rc = lib.bgt_track_turns_device_noalloc(els, len(lat.elements), C.byref(sp), v.data_ptr(), b.data_ptr(),
                                            s.data_ptr(), ie.data_ptr(), it.data_ptr(), b.numel(), 0, 3,
                                            C.byref(skip), 0, None, status.data_ptr(), err, 256)
    assert rc == 0, err.value.decode()
    torch.cuda.synchronize()
    assert int(status.item()) == 1
    assert torch.equal(v, torch.tensor(v0, dtype=torch.float64, device="cuda"))
    _noalloc(torch, lat, a, 3)  # asserts status 0
    r = _device_arrays(torch, v0, lat)
    _regular(torch, lat, r, 3)
    for x, y in zip(a, r):
        assert torch.equal(x, y)
