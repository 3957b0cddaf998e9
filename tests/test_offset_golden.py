"""offset_particle (bmad/code/offset_particle.f90) against the reference's
regression_tests/coord_test/output.correct, forward rows (orientation 1,
direction 1): the misaligned bends B1 (offsets, pitches, roll) and B2 (plus
ref_tilt) set into the body frame and back, drifting to the edges or at a
given s, with track1 through the aligned bend between set and unset; and
the misaligned solenoid Q1, whose offset_particle is that of any straight
element (a drift with the same misalignment stands in for it; its solenoid
body is outside the path).  Elements restate
regression_tests/coord_test/coord_test.bmad (line l2, electrons at
E_tot = 1e8).  The rows print 8 decimals; the tolerance is their ABS 1e-8.
"""
from __future__ import annotations

import ctypes as C
import json
from pathlib import Path

import pytest

from bgt import lattice as L
from oracle import oracle as O

GOLD = json.loads((Path(__file__).parent / "golden" / "reference_golden.json").read_text())["coord"]
E_TOT = 1e8
MIS = {"x_offset": 0.2, "y_offset": 0.3, "x_pitch": 0.1, "y_pitch": 0.2}


def _row(name, step):
    return GOLD[f"{name}:O:1:D:1:{step}-orb"]


def _ele(key, values, lib):
    e = L.Element(key, "E", dict(values))
    lat = L.Lattice([e], L.Species("electron", L.M_ELECTRON, -1), L.p0c_from_e_tot(E_TOT, L.M_ELECTRON), E_TOT)
    lat.finalize()
    return O.to_ele(lat.elements[0], lib), lat.p0c


ELEMENTS = {
    "Q1": ("drift", dict(l=2.0, tilt=2.0, **MIS)),
    "B0": ("sbend", dict(l=2.0, g=0.1, dg=-0.1)),
    "B1": ("sbend", dict(l=2.0, g=0.1, dg=-0.1, roll=0.3, **MIS)),
    "B2": ("sbend", dict(l=2.0, g=0.1, dg=-0.1, roll=0.3, ref_tilt=2.0, **MIS)),
}


def _aligned(name):
    # the element after zero_ele_offsets (bmad/code/zero_ele_offsets.f90):
    # no offsets, pitches, tilt, roll or ref_tilt -- coord_test restores a
    # bend's ref_tilt only after this track1
    key, v = ELEMENTS[name]
    drop = ("x_offset", "y_offset", "x_pitch", "y_pitch", "roll", "tilt", "ref_tilt")
    return key, {k: x for k, x in v.items() if k not in drop}


def _coord(vec, p0c, lib):
    orb = O.Coord()
    v = (C.c_double * 6)(*vec)
    lib.bgo_init_coord(C.byref(orb), v, p0c, C.byref(O.make_param(L.M_ELECTRON, -1)))
    return orb


def _check(what, orb, row, s_out=None):
    for i in range(6):
        assert abs(orb.vec[i] - row["values"][i]) <= row["tol"], (what, i, orb.vec[i], row["text"][i])
    if s_out is not None:
        assert abs(s_out - row["values"][7]) <= row["tol"], (what, "s_out", s_out, row["text"][7])


@pytest.mark.parametrize("name", ["B0", "B1", "B2"])
def test_drift_to_edges_and_track(name, oracle_lib):
    lib = oracle_lib
    ele, p0c = _ele(*ELEMENTS[name], lib)
    ele2, _ = _ele(*_aligned(name), lib)
    param = O.make_param(L.M_ELECTRON, -1)
    orb = _coord(_row(name, "Drift-Start")["values"][:6], p0c, lib)
    s = C.c_double()
    lib.bgo_offset_particle(C.byref(ele), 1, C.byref(orb), 0, 0.0, C.byref(param), C.byref(s))
    _check(f"{name} set", orb, _row(name, "Drift-In:"), s.value)
    lib.bgo_track1(C.byref(orb), C.byref(ele2), C.byref(param))
    _check(f"{name} track", orb, _row(name, "Drift-Xfer"))
    lib.bgo_offset_particle(C.byref(ele), 0, C.byref(orb), 0, 0.0, C.byref(param), C.byref(s))
    _check(f"{name} unset", orb, _row(name, "Drift-Out"), s.value)


@pytest.mark.parametrize("variant", ["glibc", "cr"])
@pytest.mark.parametrize("name", ["Q1", "B0", "B1", "B2"])
def test_at_a_given_s(name, variant, oracle_lib):
    # the "cr" build takes the arc shift by the particle-dependent angle with
    # correctly rounded transcendentals, as the device's moving bend
    # apertures do
    lib = oracle_lib if variant == "glibc" else O.load(variant="cr")
    ele, p0c = _ele(*ELEMENTS[name], lib)
    param = O.make_param(L.M_ELECTRON, -1)
    start = _row(name, "Static-Start")
    orb = _coord(start["values"][:6], p0c, lib)
    s = C.c_double()
    lib.bgo_offset_particle(C.byref(ele), 1, C.byref(orb), 1, start["values"][7], C.byref(param), C.byref(s))
    _check(f"{name} set at s", orb, _row(name, "Static-In"), s.value)
    lib.bgo_offset_particle(C.byref(ele), 0, C.byref(orb), 1, s.value, C.byref(param), C.byref(s))
    _check(f"{name} unset at s", orb, _row(name, "Static-Out"), s.value)


def test_straight_element_set_drifting_to_the_edge(oracle_lib):
    lib = oracle_lib
    ele, p0c = _ele(*ELEMENTS["Q1"], lib)
    param = O.make_param(L.M_ELECTRON, -1)
    orb = _coord(_row("Q1", "Drift-Start")["values"][:6], p0c, lib)
    s = C.c_double()
    lib.bgo_offset_particle(C.byref(ele), 1, C.byref(orb), 0, 0.0, C.byref(param), C.byref(s))
    _check("Q1 set", orb, _row("Q1", "Drift-In:"), s.value)
