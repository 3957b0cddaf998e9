"""Pin the CPU oracle to the reference's own golden vectors
(tests/golden/reference_golden.json, extracted by tests/golden/make_golden.py
from the reference's regression_tests/*/output.correct).

Element inputs are restated from
regression_tests/tracking_method_test/tracking_method_test.bmad:9-141,
regression_tests/fringe_test/fringe_test.bmad and
regression_tests/aperture_test/aperture_test.{bmad,f90}.
Each comparison allows the row's own ABS tolerance or half a unit in the last
printed digit of the golden value, whichever is larger.
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from bgt import lattice as L
from oracle import oracle as O

GOLD = json.loads((Path(__file__).parent / "golden" / "reference_golden.json").read_text())
PI = L.PI
E_TOT = 1e6  # tracking_method_test.bmad:141, fringe_test.bmad:2
# tracking_method_test.bmad sets no parameter[particle], so it tracks Bmad's
# default species, the positron; fringe_test.bmad sets Electron.
POSITRON = L.Species("positron", L.M_ELECTRON, +1)
START = [1e-3, 2e-3, 3e-3, 4e-3, 5e-3, 6e-3]  # tracking_method_test.bmad:9-14


def tol_of(text: str, abs_tol: float) -> float:
    mant, _, exp = text.upper().partition("E")
    digits = len(mant.split(".")[1]) if "." in mant else 0
    unit = 10.0 ** (int(exp or 0) - digits)
    return max(abs_tol, 0.5 * unit * 1.0001)


def check_row(name, got, row, idx=range(6)):
    for i in idx:
        tol = tol_of(row["text"][i], row["tol"])
        assert abs(got[i] - row["values"][i]) <= tol, f"{name}[{i}]: {got[i]!r} vs {row['values'][i]} (tol {tol})"


def q0(**kw):
    # q0: quadrupole, a0 = 0.01, a1 = 0.1, vkick = -0.0001, b0_elec = -2e3, a1_elec = 2e4
    vals = {"vkick": -0.0001}
    vals.update(kw)
    return dict(values=vals, a_pole={0: 0.01, 1: 0.1}, a_pole_elec={1: 2e4}, b_pole_elec={0: -2e3})


def sb0(**kw):
    # sb0 / rb0: bend, a0 = 0.01, a1 = 0.1, vkick = -0.0001, b0_elec = -2e3,
    # a1_elec = 2e4, r0_mag = 2, r0_elec = 3 (tracking_method_test.bmad:79-80)
    vals = {"vkick": -0.0001, "r0_mag": 2.0, "r0_elec": 3.0}
    vals.update(kw)
    return dict(values=vals, a_pole={0: 0.01, 1: 0.1}, a_pole_elec={1: 2e4}, b_pole_elec={0: -2e3})


# name -> (key, values, extra Element kwargs)
ELEMENTS = {
    "DRIFT1": ("drift", {"l": 4.5, "x_offset": 0.05, "y_pitch": 0.001, "tilt": 0.1}, {"num_steps": 10}),
    "INSTRUMENT1": ("instrument", {"l": 4.5}, {"num_steps": 10}),
    "MONITOR1": ("monitor", {"l": 4.5}, {"num_steps": 10}),
    "RCOLLIMATOR1": ("rcollimator", {"l": 4.5, "x1_limit": 0.2, "x2_limit": 0.2, "y1_limit": 0.1, "y2_limit": 0.1,
                                     "x_offset": 0.02, "y_pitch": 0.001, "tilt": 0.1}, {"num_steps": 10}),
    "ECOLLIMATOR1": ("ecollimator", {"l": 4.5, "x1_limit": 0.2, "x2_limit": 0.2, "y1_limit": 0.1, "y2_limit": 0.1,
                                     "x_offset": 0.02, "y_pitch": 0.001, "tilt": 0.1, "hkick": 0.01,
                                     "vkick": 0.002}, {"num_steps": 10}),
    "HKICKER1": ("hkicker", {"l": 4.5, "kick": 0.005, "x_offset": 0.05, "y_pitch": 0.001, "tilt": 0.1},
                 {"num_steps": 10}),
    "VKICKER1": ("vkicker", {"l": 4.5, "kick": 0.005, "x_offset": 0.05, "y_pitch": 0.001, "tilt": 0.1},
                 {"num_steps": 10}),
    "KICKER1": ("kicker", {"l": 4.5, "vkick": 0.003, "x_offset": 0.05, "y_pitch": 0.001, "tilt": 0.1},
                {"num_steps": 10, "b_pole": {0: 0.002}}),
    "OCTUPOLE1": ("octupole", {"l": 4.5, "k3": 1e3, "tilt": PI / 8, "x_offset": 0.01, "y_pitch": 0.001},
                  {"num_steps": 10}),
    "SEXTUPOLE1": ("sextupole", {"l": 0.6, "k2": 1.0, "tilt": PI / 6, "x_offset": 0.05, "y_pitch": 0.001},
                   {"num_steps": 10}),
    "THICK_MULTIPOLE1": ("thick_multipole", {"l": 4.5, "x_offset": 0.02, "tilt": 0.1},
                         {"a_pole": {2: 1.0}, "b_pole": {3: 20.0}}),
    "AB_MULTIPOLE1": ("ab_multipole", {"x_offset": 0.02, "tilt": 0.1}, {"a_pole": {2: 1e2}, "b_pole": {2: 1e2}}),
    "MULTIPOLE1": ("multipole", {"x_offset": 0.05}, {"a_pole": {1: 1.0, 3: 4.5}, "b_pole": {1: PI / 4, 3: 0.31 * PI}}),
    "RFCAVITY1": ("rfcavity", {"l": 4.5, "rf_frequency": 500e6, "voltage": 1e5, "phi0": 0.1, "x_offset": 0.05,
                               "y_pitch": 0.001, "tilt": 0.1}, {"num_steps": 10}),
    # cavity_type = traveling_wave (tracking_method_test.bmad:71-72) changes
    # nothing in bmad_standard rfcavity tracking; the coupler kick does
    "RFCAVITY2": ("rfcavity", {"l": 4.5, "rf_frequency": 500e6, "voltage": 1e5, "phi0": 0.1, "x_offset": 0.05,
                               "y_pitch": 0.001, "tilt": 0.1, "coupler_strength": 0.1},
                  {"num_steps": 10, "coupler_at": "both_ends"}),
    "RFCAVITY3": ("rfcavity", {"rf_frequency": 500e6, "voltage": 1e5, "phi0": 0.1, "x_offset": 0.05,
                               "y_pitch": 0.001, "tilt": 0.1}, {"num_steps": 10, "a_pole": {2: 0.02}}),
}
# tracking_method_test.bmad:84-91 (the rows without exact multipoles):
# misaligned bends with ref_tilt, electric multipoles; RBEND4 and SBEND5 with
# the exact (PTC) bend edge of fringe_type full
for _n, _key, _b, _fr in (
        ("SBEND3", "sbend", sb0(l=0.6, k1=0.3, k2=3.0, x_offset=0.05, y_pitch=0.001, ref_tilt=0.1), None),
        ("RBEND4", "rbend", sb0(l=0.6, g=0.01, dg=-0.0099, e1=0.1, e2=0.2, x_offset=0.05, y_pitch=0.001,
                                ref_tilt=0.1), "full"),
        ("SBEND5", "sbend", sb0(l=0.6, g=0.01, e1=0.1, e2=0.2, x_offset=0.05, y_pitch=0.001, ref_tilt=0.1,
                                fint=0.7, hgap=2.0), "full"),
        ("RBEND6", "rbend", sb0(l=0.6, g=0.01, dg=-0.0099999, e1=0.1, e2=0.2, x_offset=0.05, y_pitch=0.001,
                                ref_tilt=0.1), None),
        ("SBEND7", "sbend", sb0(l=0.6, g=0.01, e1=0.1, e2=0.2, x_offset=0.05, y_pitch=0.001, ref_tilt=0.1),
         None)):
    _kw = dict(num_steps=10, **_b)
    if _fr:
        _kw["fringe_type"] = _fr
    ELEMENTS[_n] = (_key, _kw.pop("values"), _kw)
for _n, _k1, _fr in (("QUADRUPOLE1", 1.0, None), ("QUADRUPOLE2", -1.0, None), ("QUADRUPOLE3", 1e-20, None),
                     ("QUADRUPOLE4", 1.0, "full"), ("QUADRUPOLE5", -1.0, "full")):
    _q = q0(l=0.6, k1=_k1, tilt=PI / 4, x_offset=0.05, y_pitch=0.001)
    _kw = dict(num_steps=10, **_q)
    _kw.pop("values")
    if _fr:
        _kw["fringe_type"] = _fr
    ELEMENTS[_n] = ("quadrupole", _q["values"], _kw)


def make_element(name):
    key, vals, kw = ELEMENTS[name]
    kw = dict(kw)
    e = L.Element(key, name, dict(vals), **kw)
    lat = L.Lattice([e], POSITRON, L.p0c_from_e_tot(E_TOT, L.M_ELECTRON), E_TOT)
    lat.finalize()
    return lat


@pytest.mark.parametrize("name", sorted(ELEMENTS))
def test_tracking_method_bmad_standard(name, oracle_lib):
    lat = make_element(name)
    ele = O.to_ele(lat.elements[0], oracle_lib)
    param = O.make_param(L.M_ELECTRON, +1)
    vec, beta, state = O.track1(ele, START, lat.p0c, param, lib=oracle_lib)
    assert state == L.ALIVE
    check_row(name, vec, GOLD["tracking_method"][name])


@pytest.mark.parametrize("name", sorted(ELEMENTS))
def test_tracking_method_time_column(name, oracle_lib):
    """The rows' seventh column checks the particle time t against z: the
    change of z less c_light times the change of beta * (reference time - t)
    (tracking_method_test.f90:219-221), a residual of order 1e-16 when t
    advances as the reference advances it and of order the element length
    when it does not.  The oracle carries t in quad precision."""
    from helpers import time_residual

    lat = make_element(name)
    e = lat.elements[0]
    ele = O.to_ele(e, oracle_lib)
    param = O.make_param(L.M_ELECTRON, +1)
    vec, beta, state, beta0, t0, t1 = O.track1_timed(ele, START, lat.p0c, param, lib=oracle_lib)
    assert state == L.ALIVE
    d = time_residual(START[4], vec[4], beta0, beta, t0, t1, e.v("ref_time_start"), e.v("delta_ref_time"))
    check_row(name, list(vec) + [d], GOLD["tracking_method"][name], idx=range(7))


@pytest.mark.parametrize("name", sorted(set(ELEMENTS) & set(GOLD["tracking_method_abs_time"])))
def test_tracking_method_absolute_time(name, oracle_lib):
    """The "-Abs_Time" rows: the RF cavities tracked with
    bmad_com%absolute_time_tracking = T (tracking_method_test.f90:113-119,
    174-179), the RF phase from the particle time t less the cavity's
    ref_time_start (particle_rf_time.f90:74-76) folded in quad precision."""
    from helpers import time_residual

    lat = make_element(name)
    e = lat.elements[0]
    ele = O.to_ele(e, oracle_lib)
    param = O.make_param(L.M_ELECTRON, +1, absolute_time=True)
    vec, beta, state, beta0, t0, t1 = O.track1_timed(ele, START, lat.p0c, param, lib=oracle_lib)
    assert state == L.ALIVE
    d = time_residual(START[4], vec[4], beta0, beta, t0, t1, e.v("ref_time_start"), e.v("delta_ref_time"))
    check_row(name + "-Abs_Time", list(vec) + [d], GOLD["tracking_method_abs_time"][name], idx=range(7))


def test_fringe_hwang_edges(oracle_lib):
    # fringe_test.bmad: b: sbend, e1 = 0.1, e2 = -0.2, k1 = 0.1, g = 0.1, fint = 0.5, hgap = 0.4
    e = L.Element("sbend", "B", {"l": 0.0, "e1": 0.1, "e2": -0.2, "k1": 0.1, "g": 0.1, "fint": 0.5, "hgap": 0.4})
    lat = L.Lattice([e], L.Species("electron", L.M_ELECTRON, -1), L.p0c_from_e_tot(E_TOT, L.M_ELECTRON), E_TOT)
    lat.finalize()
    ele = O.to_ele(lat.elements[0], oracle_lib)
    start = [0.01, 0.02, 0.03, 0.04, 0.0, 0.5]
    param = O.make_param(L.M_ELECTRON, -1)
    for entering, row in ((1, "Up-Orb"), (0, "Dn-Orb")):
        c = O.Coord()
        v = (O.C.c_double * 6)(*start)
        oracle_lib.bgo_init_coord(O.C.byref(c), v, lat.p0c, O.C.byref(param))
        oracle_lib.bgo_hwang_bend_edge_kick(O.C.byref(ele), entering, O.C.byref(c), O.C.byref(param))
        d = [c.vec[i] - start[i] for i in range(6)]
        check_row(row, d, GOLD["fringe"][row])


def _collimator(key):
    # aperture_test.bmad: ec / rc (same attributes)
    vals = dict(px_aperture_width2=0.01, px_aperture_center=0.01, py_aperture_width2=0.015,
                z_aperture_width2=0.2, z_aperture_center=-0.6, pz_aperture_width2=0.03, pz_aperture_center=0.02,
                x1_limit=1e-10, x2_limit=0.02, y1_limit=0.015, y2_limit=0.015)
    e = L.Element(key, key.upper()[:2], {k: v for k, v in vals.items() if not k.startswith(("px", "py", "z_", "pz"))})
    lat = L.Lattice([e], L.Species("antimuon", 105.6583755e6, 1), 3.094353005e9, 0.0)
    lat.finalize()
    o = O.to_ele(lat.elements[0])
    for k, v in vals.items():
        setattr(o, k, v)
    return o


def f32(v):
    """aperture_test.f90 assigns single-precision literals (0.01, 1e-5, ...)
    to its real(rp) stencil variables."""
    return float(np.float32(v))


STENCILS = {
    # (fixed coords, index pair varied, (x0, xw2), (y0, yw2)) -- aperture_test.f90:66-140
    "Pxy": (lambda a, b: [0.0, a, 0.0, b, -0.6, 0.02], (f32(0.01), f32(0.01)), (0.0, f32(0.015))),
    "xy": (lambda a, b: [a, 0.1, b, 0.0, -0.6, 0.02], (f32(0.01), f32(0.01)), (0.0, f32(0.015))),
    "zPz": (lambda a, b: [0.0, 0.01, 0.0, 0.0, a, b], (f32(-0.6), f32(0.2)), (f32(0.02), f32(0.03))),
}


@pytest.mark.parametrize("elem", ["EC", "RC"])
@pytest.mark.parametrize("stencil", ["Pxy", "xy", "zPz"])
@pytest.mark.parametrize("sign", ["-", "+"])
def test_aperture_states(elem, stencil, sign, oracle_lib):
    ele = _collimator("ecollimator" if elem == "EC" else "rcollimator")
    mk, (x0, xw2), (y0, yw2) = STENCILS[stencil]
    eps = f32(1e-5)
    states, uf = [], []
    for i in (-1, 0, 1):
        for j in (-1, 0, 1):
            if stencil == "xy" and sign == "+":
                vec = [x0 + i * (xw2 + eps), 0.0, y0 + j * (yw2 + eps), 0.0, -0.6, 0.02]
            else:
                d = (xw2 - eps) if sign == "-" else (xw2 + eps)
                e2 = (yw2 - eps) if sign == "-" else (yw2 + eps)
                vec = mk(x0 + i * d, y0 + j * e2)
            c = O.Coord()
            for k in range(6):
                c.vec[k] = vec[k]
            c.state = 1
            c.p0c = 3.094353005e9
            c.beta = 1.0
            param = O.make_param(105.6583755e6, 1)
            oracle_lib.bgo_check_aperture_limit(O.C.byref(c), O.C.byref(ele), 1, O.C.byref(param))
            states.append(c.state)
            uf.append(param.unstable_factor)
    srow = GOLD["aperture"][f"{elem}_S_{stencil}{sign}"]
    urow = GOLD["aperture"][f"{elem}_U_{stencil}{sign}"]
    assert states == [int(v) for v in srow["values"]]
    for k in range(9):
        assert abs(uf[k] - urow["values"][k]) <= tol_of(urow["text"][k], urow["tol"]), (k, uf[k], urow["values"][k])
