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


def _noalloc(torch, lat, arrays, turns):
    lib = _lib.load()
    els = (_lib.BgtElement * len(lat.elements))(*[_lib.to_bgt_element(e) for e in lat.elements])
    sp = _lib.BgtSpecies(lat.species.mass, lat.species.charge, 1, 1e3)
    v, b, s, ie, it = arrays
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream()
    rc = lib.bgt_track_turns_device_noalloc(els, len(lat.elements), C.byref(sp), v.data_ptr(), b.data_ptr(),
                                            s.data_ptr(), ie.data_ptr(), it.data_ptr(), b.numel(), 0, turns, None,
                                            0, C.c_void_p(stream.cuda_stream), err, 256)
    assert rc == 0, err.value.decode()
    torch.cuda.synchronize()


def _regular(torch, lat, arrays, turns):
    tr = Tracker(lat)
    tr.track_turns_device(*arrays, turns)
    torch.cuda.synchronize()


@pytest.mark.parametrize("dummy", [0])
def test_noalloc_matches_regular_entry_point_twice(dummy):
    torch = pytest.importorskip("torch")
    cases = [
        (rings.fodo_ring(apertures=True), rings.BeamSpec(3000, 4e-6, 2e-6, 3e-3, 2e-3, seed=91), 25),
        (rings.error_variants(1, seed=9)[0], rings.BeamSpec(2000, 1e-6, 5e-7, 3e-3, 1e-3, seed=92), 10),
    ]
    for lat, spec, turns in cases:  # two calls in a row through the same scratch array
        v0 = rings.gaussian_beam(spec)
        a = _device_arrays(torch, v0, lat)
        _noalloc(torch, lat, a, turns)
        r = _device_arrays(torch, v0, lat)
        _regular(torch, lat, r, turns)
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
                                            s.data_ptr(), ie.data_ptr(), None, 1, 0, 1, None, 0, None, err, 256)
    assert rc == _lib.BGT_ETOOLARGE, (rc, err.value)
    assert b"scratch array holds" in err.value
