"""Momentum-aperture search (bgt.momentum_aperture): the vectorised search
state machine against a line-by-line scalar restatement of binary_search
(bsim/aperture_by_tracking/aperture_by_tracking_mod.f90:275-345), and the
rotated rings used as per-slice variants."""
from __future__ import annotations

import numpy as np

from bgt import momentum_aperture as MA
from bgt import rings


def _scalar_search(is_lost, first_guess, target):
    high_found = low_found = bracket = False
    last_high = last_low = 0.0
    accuracy = 10.0
    d = first_guess
    while accuracy > target:
        lost = is_lost(d)
        if not bracket:
            if lost:
                high_found = True
                last_high = d
                if not low_found:
                    d = d / 2.0
            else:
                low_found = True
                last_low = d
                if not high_found:
                    d = d * 2.0
            bracket = high_found and low_found
            accuracy = 10.0
        if bracket:
            if lost:
                last_high = d
                d = d - abs(d - last_low) / 2.0
            else:
                last_low = d
                d = d + abs(last_high - d) / 2.0
            accuracy = abs(last_high - last_low) / min(abs(last_high), abs(last_low))
        if abs(d) > 1.0:
            accuracy = 0.0
            last_high, last_low = 1.1, 0.9
        if abs(d) < 1.0e-6:
            accuracy = 0.0
            last_high, last_low = 2.0e-6, 0.0
    return d


def test_vectorised_search_equals_scalar_binary_search():
    thr_pos = np.array([0.0123, 0.0004, 0.7, 3.0, 2e-7, 0.02])
    thr_neg = np.array([0.011, 0.0301, 0.5, 0.3, 0.0009, 5e-7])
    orbits = np.zeros((len(thr_pos), 6))

    def lost_fn(v6, var):
        pz = v6[5]
        return np.where(pz >= 0, pz > thr_pos[var], -pz > thr_neg[var])

    for guess, target in ((0.001, 0.01), (0.05, 1e-4)):
        ap, steps = MA.search(lost_fn, orbits, guess, target)
        for i in range(len(thr_pos)):
            assert ap[i, 0] == _scalar_search(lambda d: d > thr_pos[i], guess, target)
            assert ap[i, 1] == -_scalar_search(lambda d: d > thr_neg[i], guess, target)
        assert steps > 5


def test_rotated_ring_keeps_element_indices():
    lat = rings.fodo_ring(apertures=True)
    r = MA.rotated(lat, 100)
    assert len(r) == len(lat)
    assert [e.ix_ele for e in r.elements] == [e.ix_ele for e in lat.elements[100:] + lat.elements[:100]]
    assert [e.key for e in r.elements[:3]] == [e.key for e in lat.elements[100:103]]
    assert abs(r.circumference - lat.circumference) < 1e-9


def test_closed_orbit_at_tracks_in_order():
    calls = []

    def one_pass(v, b, e):
        calls.append((b, e))
        return v + (e - b)

    out = MA.closed_orbit_at(one_pass, np.zeros(6), [0, 3, 3, 10])
    assert calls == [(0, 3), (3, 10)]
    assert np.all(out[:, 0] == [0, 3, 3, 10])
