"""Resuming from a checkpoint reproduces an uninterrupted run bit for bit
(losses included): the tracker's restart contract (turn0)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_resume_from_checkpoint_is_bit_identical(tmp_path):
    from bgt import beam_io as B
    from bgt import rings
    from bgt.track import Tracker

    lat = rings.fodo_ring(apertures=True)
    tr = Tracker(lat)
    v0 = rings.gaussian_beam(rings.CONFIG1_BEAM, n=20000)
    v0[0:4] *= 7.0  # large amplitudes: part of the bunch hits the apertures
    full = tr.make_bunch(v0.copy())
    tr.track_turns(full, 30)
    part = tr.make_bunch(v0.copy())
    tr.track_turns(part, 12)
    B.save_checkpoint(str(tmp_path / "ck.npz"), part, 12)
    again, turn, _ = B.load_checkpoint(str(tmp_path / "ck.npz"))
    tr.track_turns(again, 30 - turn, turn0=turn)
    for k in ("vec6", "beta", "state", "ix_ele_lost", "ix_turn_lost"):
        assert np.array_equal(getattr(again, k), getattr(full, k)), k
    assert np.any(full.state != 1)  # the run does lose particles
