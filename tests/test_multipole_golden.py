"""multipole_ele_to_ab (bmad/code/multipole_ele_to_ab.f90), both
restatements -- the product's host conversion (bgt.lattice) that fills the
element tables and the oracle's (bgo_multipole_ele_to_ab) -- against the
reference's regression_tests/multipole_test/output.correct "MULT" rows:
a1, a3, a5, b2, b4, b6 of the magnetic multipoles with and without the
element tilt and the kick/strength terms, and the highest electric order.
The elements restate regression_tests/multipole_test/multipole.bmad (qq, bb,
mm; the elseparator ee is outside the tracker's element set).  The rows are
printed with 5 significant digits (es12.4), so a value must agree to half a
unit in that digit, and a printed zero must be zero.
"""
from __future__ import annotations

import ctypes as C
import json
import math
from pathlib import Path

import numpy as np
import pytest

from bgt import lattice as L
from oracle import oracle as O

GOLD = json.loads((Path(__file__).parent / "golden" / "reference_golden.json").read_text())["multipole"]
ELEC = dict(a_pole_elec={n: (n + 1) * 1e-2 for n in range(6)}, b_pole_elec={n: (n + 1) * 1e-3 for n in range(6)})


def _elements():
    qq = L.Element("quadrupole", "QQ", {"l": 1e-3, "k1": 0.1, "tilt": math.pi / 4}, scale_multipoles=False,
                   a_pole={n: float(n + 1) for n in range(6)}, b_pole={n: (n + 1) / 10 for n in range(6)}, **ELEC)
    # bb sets a5 twice (5, then 6) and no a4
    bb = L.Element("sbend", "BB", {"l": 1e-3, "g": 1e-2, "k1": 0.1, "k2": 0.2, "ref_tilt": math.pi / 2},
                   a_pole={0: 1.0, 1: 2.0, 2: 3.0, 3: 4.0, 5: 6.0}, b_pole={n: (n + 1) / 10 for n in range(6)},
                   **ELEC)
    mm = L.Element("multipole", "MM", {}, a_pole={6: 1.0, 1: 2.0, 2: 3.0, 3: 4.0, 4: 5.0, 5: 6.0},
                   b_pole={n: (n + 1) / 10 for n in range(6)})
    lat = L.Lattice([qq, bb, mm], L.Species("electron", L.M_ELECTRON, -1), L.p0c_from_e_tot(1e9, L.M_ELECTRON),
                    1e9, "multipole_test")
    lat.finalize()
    return {e.name: e for e in lat.elements}


def _check(name, a, b, ix_elec, row):
    got = [a[1], a[3], a[5], b[2], b[4], b[6]]
    for g, v, t in zip(got, row["values"], row["text"]):
        if v == 0:
            assert g == 0, (name, got, row["text"])
        else:
            exp = int(t.upper().split("E")[1])
            assert abs(g - v) <= 0.5e-4 * 10.0 ** exp * 1.0001, (name, got, row["text"])
    assert ix_elec == row["ix"], (name, ix_elec, row["ix"])


CASES = [(f"MULT-{iu}{ik}-{nm}", iu == 2, ik == 2, nm) for nm in ("QQ", "BB", "MM") for iu in (1, 2)
         for ik in (1, 2)]


@pytest.mark.parametrize("row,use_tilt,kicks,name", CASES)
def test_host_conversion(row, use_tilt, kicks, name):
    e = _elements()[name]
    _, a, b = L.multipole_ele_to_ab(e, use_tilt, False, kicks)
    ix_e, _, _ = L.multipole_ele_to_ab(e, use_tilt, True, kicks)
    _check(row, a, b, ix_e, GOLD[row])


@pytest.mark.parametrize("row,use_tilt,kicks,name", CASES)
def test_oracle_conversion(row, use_tilt, kicks, name, oracle_lib):
    ele = O.to_ele(_elements()[name], oracle_lib)
    a = np.zeros(O.N_POLE)
    b = np.zeros(O.N_POLE)
    ae = np.zeros(O.N_POLE)
    be = np.zeros(O.N_POLE)
    dp = C.POINTER(C.c_double)
    oracle_lib.bgo_multipole_ele_to_ab(C.byref(ele), int(use_tilt), 0, int(kicks), a.ctypes.data_as(dp),
                                       b.ctypes.data_as(dp), None)
    ix_e = oracle_lib.bgo_multipole_ele_to_ab(C.byref(ele), int(use_tilt), 1, int(kicks), ae.ctypes.data_as(dp),
                                              be.ctypes.data_as(dp), None)
    _check(row, a, b, ix_e, GOLD[row])
