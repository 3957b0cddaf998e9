"""GPU momentum aperture (all slices and signs batched as rotated-ring
variants) against the same search driven by the correctly rounded oracle:
identical apertures."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_momentum_aperture_matches_oracle():
    from bgt import da
    from bgt import momentum_aperture as MA
    from bgt import rings
    from helpers import oracle_batch_one_turn, oracle_track_elements
    from oracle import oracle as O

    lat = rings.fodo_ring(apertures=True)
    starts = [0, 5, 37, 200, 500]
    n_turns = 30
    gpu = MA.momentum_aperture(lat, starts, n_turns)

    co0 = da.variant_optics(oracle_batch_one_turn([lat]), 1).closed_orbit[0]
    sco = MA.closed_orbit_at(
        lambda v, b, e: oracle_track_elements(lat, v, b, e, 1, variant="cr")[0], co0, starts)
    lib = O.load(variant="cr")
    rots = [MA.rotated(lat, s) for s in starts]
    eles = [O.to_eles(r, lib) for r in rots]
    param = O.make_param(lat.species.mass, lat.species.charge)

    def lost_fn(v6, var):
        out = np.zeros(v6.shape[1], bool)
        for k in np.unique(var):
            idx = np.nonzero(var == k)[0]
            v = np.ascontiguousarray(v6[:, idx])
            n = v.shape[1]
            b = O.beta_of(lat.p0c, v[5], lat.species.mass)
            st = np.ones(n, np.int32)
            O.track_turns(eles[k], lat.p0c, param, v, b, st, np.full(n, -1, np.int32), np.full(n, -1, np.int32),
                          n_turns, lib=lib)
            out[idx] = st != 1
        return out

    ap, steps = MA.search(lost_fn, sco, 0.001, 0.01)
    assert np.array_equal(gpu.aperture, ap) and gpu.steps == steps
    assert np.all(gpu.aperture[:, 0] > 0) and np.all(gpu.aperture[:, 1] < 0)
