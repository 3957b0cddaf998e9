"""The host side of bgt_create -- the element-table compiler -- and the
argument checks of the C ABI, without a GPU.

bgt_create compiles every element of every variant before its first CUDA
call, so a supported lattice gets as far as the device (BGT_ECUDA on a
machine without a GPU, BGT_OK with one) while an element outside the
library's scope is rejected with BGT_EUNSUPPORTED and named on stderr --
the caller's cue to keep Bmad's own tracking for that lattice.  Calls with a
null handle or invalid sizes return BGT_EINVAL and never reach the device.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from bgt import _lib
from bgt import lattice as L
from bgt import rings

from helpers import rare_zoo_lattice, zoo_lattice


def _elements(lats):
    n_ele = len(lats[0].elements)
    arr = (_lib.BgtElement * (n_ele * len(lats)))()
    for v, lat in enumerate(lats):
        for i, e in enumerate(lat.elements):
            arr[v * n_ele + i] = _lib.to_bgt_element(e)
    return arr, n_ele


def _species(lat):
    return _lib.BgtSpecies(lat.species.mass, lat.species.charge, 1, 1e3)


def _create(lats, arr=None):
    lib = _lib.load()
    if arr is None:
        arr, n_ele = _elements(lats)
    else:
        n_ele = len(arr) // len(lats)
    sp = _species(lats[0])
    h = C.c_void_p()
    rc = lib.bgt_create(C.byref(h), arr, n_ele, len(lats), C.byref(sp), 0)
    if rc == _lib.BGT_OK:
        lib.bgt_destroy(h)
    return rc


def _reaches_device(rc):
    return rc in (_lib.BGT_OK, _lib.BGT_ECUDA)


@pytest.mark.parametrize("make", [rings.fodo_ring, zoo_lattice, rare_zoo_lattice])
def test_supported_lattices_compile(make):
    assert _reaches_device(_create([make()]))


def test_error_variants_compile():
    assert _reaches_device(_create(rings.error_variants(3, seed=1)))


def _line(key, values, **kw):
    e = L.Element(key, "X", dict(values), **kw)
    lat = L.Lattice([L.Element("drift", "D", {"l": 1.0}), e], L.Species("electron", L.M_ELECTRON, -1),
                    rings.p0c(), rings.E_TOT, "line")
    return lat.finalize()


@pytest.mark.parametrize("key,values,kw,msg", [
    ("sbend", {"l": 1.0, "g": 0.01}, {"exact_multipoles": 1}, "exact_multipoles"),
    ("drift", {"l": 1.0}, {"b_pole_elec": {1: 1e5}}, "electric multipoles"),
])
def test_unsupported_elements_are_rejected_and_named(key, values, kw, msg, capfd):
    rc = _create([_line(key, values, **kw)])
    err = capfd.readouterr().err
    assert rc == _lib.BGT_EUNSUPPORTED
    assert "ix_ele=2" in err and msg in err, err


def test_unknown_key_and_momentum_mismatch_are_rejected(capfd):
    lat = _line("drift", {"l": 1.0})
    arr, _ = _elements([lat])
    arr[1].key = 99
    assert _create([lat], arr) == _lib.BGT_EUNSUPPORTED
    assert "key 99" in capfd.readouterr().err
    arr, _ = _elements([lat])
    arr[1].p0c = arr[1].p0c * (1 + 1e-12)
    assert _create([lat], arr) == _lib.BGT_EUNSUPPORTED
    assert "p0c" in capfd.readouterr().err


def test_rf_without_frequency_is_invalid(capfd):
    rc = _create([_line("rfcavity", {"l": 0.5, "voltage": 1e6})])
    assert rc == _lib.BGT_EINVAL
    assert "rf_frequency" in capfd.readouterr().err


def test_create_checks_its_arguments():
    lats = [rings.fodo_ring(), rings.fodo_ring()]
    arr, n_ele = _elements(lats)
    lib = _lib.load()
    sp = _species(lats[0])
    h = C.c_void_p()
    assert lib.bgt_create(C.byref(h), arr, 0, 2, C.byref(sp), 0) == _lib.BGT_EINVAL
    assert lib.bgt_create(C.byref(h), arr, n_ele, 0, C.byref(sp), 0) == _lib.BGT_EINVAL
    assert lib.bgt_create(None, arr, n_ele, 2, C.byref(sp), 0) == _lib.BGT_EINVAL
    assert lib.bgt_create(C.byref(h), arr, n_ele, 2, None, 0) == _lib.BGT_EINVAL


def test_null_handle_calls_return_einval():
    lib = _lib.load()
    v = np.zeros(6, np.float64)
    b = np.ones(1, np.float64)
    s = np.ones(1, np.int32)
    i = np.zeros(1, np.int32)
    dp = _lib.ptr(v, C.c_double)
    bp = _lib.ptr(b, C.c_double)
    sp = _lib.ptr(s, C.c_int32)
    ip = _lib.ptr(i, C.c_int32)
    assert lib.bgt_track_turns(None, dp, bp, None, sp, ip, ip, None, 1, 0, 1) == _lib.BGT_EINVAL
    assert lib.bgt_track_elements(None, dp, bp, None, sp, ip, None, 1, 0, 1) == _lib.BGT_EINVAL
    t = _lib.BgtTuning(128, 4, 0, 0, 0)
    assert lib.bgt_set_tuning(None, C.byref(t)) == _lib.BGT_EINVAL
    assert lib.bgt_get_tuning(None, C.byref(t)) == _lib.BGT_EINVAL
    assert lib.bgt_table_info(None, None, None) == _lib.BGT_EINVAL
    assert lib.bgt_kernel_launch_count(None) == -1
    assert lib.bgt_last_error(None) == b"null handle"
    assert lib.bgt_device_status(None, None) == _lib.BGT_EINVAL
    assert lib.bgt_da_scan_grid(None, dp, 1, 1, 4, 0.0, 1.0, 8, 0.01, 1.0, 10, dp, None) == _lib.BGT_EINVAL
    assert lib.bgt_destroy(None) == 0


def test_error_messages_are_per_thread():
    """bgt_last_error returns the message of the last failed call on the
    calling thread: a failure on another thread does not replace it."""
    import threading

    lib = _lib.load()
    t = _lib.BgtTuning(128, 4, 0, 0, 0)
    assert lib.bgt_get_tuning(None, C.byref(t)) == _lib.BGT_EINVAL
    mine = lib.bgt_last_error(None)
    other = []

    def worker():
        lib.bgt_track_elements(None, None, None, None, None, None, None, 1, 0, 1)
        other.append(lib.bgt_last_error(None))

    th = threading.Thread(target=worker)
    th.start()
    th.join()
    assert other and other[0] != mine
    assert lib.bgt_last_error(None) == mine


def test_noalloc_checks_arguments_first():
    lib = _lib.load()
    lat = rings.fodo_ring()
    arr, n_ele = _elements([lat])
    sp = _species(lat)
    buf = C.create_string_buffer(256)
    # no particle buffers: rejected before any device call
    rc = lib.bgt_track_turns_device_noalloc(arr, n_ele, C.byref(sp), None, None, None, None, None, 10, 0, 1,
                                             None, 0, None, None, buf, 256)
    assert rc == _lib.BGT_EINVAL and b"invalid argument" in buf.value
    # a launch shape without a kernel instance, or a bad tuning value, is
    # refused before any device call (the pointers below are never read)
    fake = C.c_void_p(16)
    for tun, what in ((_lib.BgtTuning(64, 8, 0, 0, 0), b"tuning must be"),
                      (_lib.BgtTuning(128, 4, 0, -1, 0), b"invalid tuning"),
                      (_lib.BgtTuning(256, 2, 0, 0, 0, 0, 2), b"invalid tuning")):
        rc = lib.bgt_track_turns_device_noalloc(arr, n_ele, C.byref(sp), fake, fake, fake, fake, None, 10, 0, 1,
                                                 C.byref(tun), 0, None, None, buf, 256)
        assert rc == _lib.BGT_EINVAL and what in buf.value, buf.value
