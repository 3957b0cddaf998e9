"""The device tracker against the reference's own golden vectors:
regression_tests/tracking_method_test/output.correct "Bmad_Standard" rows,
each element tracked by the GPU through the C ABI (track1 of a one-element
lattice), within the row's tolerance -- and bit-identical to the correctly
rounded oracle on the same element.  QUADRUPOLE1-3 carry electric
multipoles (kicks that change the energy, electric longitudinal fringe)."""
from __future__ import annotations

import numpy as np
import pytest

from test_oracle_golden import ELEMENTS, GOLD, START, check_row, make_element

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(ELEMENTS))
def test_gpu_reproduces_golden_row(name):
    from bgt.track import Tracker
    from helpers import oracle_track_elements

    lat = make_element(name)
    tr = Tracker(lat)
    v0 = np.array(START, dtype=np.float64).reshape(6, 1)
    b = tr.make_bunch(v0.copy())
    tr.track_turns(b, 1)
    assert b.state[0] == 1
    check_row(name, b.vec6[:, 0], GOLD["tracking_method"][name])
    ov, ob, ost, _, _ = oracle_track_elements(lat, v0.copy(), 0, 1, 1, variant="cr")
    assert np.array_equal(b.vec6, ov) and np.array_equal(b.beta, ob)


@pytest.mark.parametrize("name", sorted(ELEMENTS))
def test_gpu_time_column(name):
    """The rows' seventh column (the time residual, test_oracle_golden) from
    the device's particle time, which equals the oracle's quad-precision
    time bit for bit."""
    from bgt.track import Tracker
    from helpers import oracle_track_timed, time_residual

    lat = make_element(name)
    e = lat.elements[0]
    tr = Tracker(lat)
    v0 = np.array(START, dtype=np.float64).reshape(6, 1)
    b = tr.make_bunch(v0.copy(), with_time=True)
    t0, beta0 = b.t.copy(), b.beta[0]
    tr.track_turns(b, 1)
    d = time_residual(START[4], b.vec6[4, 0], beta0, b.beta[0], t0[0], b.t[0], e.v("ref_time_start"),
                      e.v("delta_ref_time"))
    check_row(name, list(b.vec6[:, 0]) + [d], GOLD["tracking_method"][name], idx=range(7))
    ov, ob, ost, _, _, ot = oracle_track_timed(lat, v0.copy(), 0, 1, 1)
    assert np.array_equal(b.vec6, ov) and np.array_equal(b.t, ot)


@pytest.mark.parametrize("name", sorted(set(ELEMENTS) & set(GOLD["tracking_method_abs_time"])))
def test_gpu_absolute_time_rows(name):
    """The "-Abs_Time" RF rows on the device: the phase from the particle
    time (binary128 in software), coordinates and time residual within the
    rows' tolerance and bit for bit equal to the oracle."""
    from bgt.track import Tracker
    from helpers import oracle_track_timed, time_residual

    lat = make_element(name)
    e = lat.elements[0]
    tr = Tracker(lat, absolute_time=True)
    v0 = np.array(START, dtype=np.float64).reshape(6, 1)
    b = tr.make_bunch(v0.copy())
    t0, beta0 = b.t.copy(), b.beta[0]
    tr.track_turns(b, 1)
    d = time_residual(START[4], b.vec6[4, 0], beta0, b.beta[0], t0[0], b.t[0], e.v("ref_time_start"),
                      e.v("delta_ref_time"))
    check_row(name + "-Abs_Time", list(b.vec6[:, 0]) + [d], GOLD["tracking_method_abs_time"][name], idx=range(7))
    ov, ob, ost, _, _, ot = oracle_track_timed(lat, v0.copy(), 0, 1, 1, absolute_time=True)
    assert np.array_equal(b.vec6, ov) and np.array_equal(b.t, ot)
