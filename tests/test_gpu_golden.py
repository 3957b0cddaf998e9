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
