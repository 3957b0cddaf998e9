"""The BEAM-mode turn loop (bgt.ltt.run_beam_mode) against a turn-by-turn
restatement of ltt_run_beam_mode (bsim/modules/lt_tracking_mod.f90:
1571-1719), both driving the CPU oracle as the tracker: the same stop turn and
reason, live count, dead-count reports, output turns and final particles,
whether the stop falls on a segment end or inside one."""
from __future__ import annotations

import math

import numpy as np
import pytest

from bgt import lattice as L
from bgt import ltt, rings
from bgt.track import Bunch
from oracle import oracle as O


class OracleTracker:
    """track_turns(bunch, n_turns, turn0) on the CPU oracle."""

    def __init__(self, lat, lib):
        self.lat = lat
        self.lib = lib
        self.eles = O.to_eles(lat, lib)
        self.param = O.make_param(lat.species.mass, lat.species.charge)
        self.calls = 0

    def track_turns(self, b, n_turns, turn0=0):
        self.calls += 1
        O.track_turns(self.eles, self.lat.p0c, self.param, b.vec6, b.beta, b.state, b.ix_ele_lost, b.ix_turn_lost,
                      n_turns, turn0=turn0, lib=self.lib)


def _nint(x):
    return int(math.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)


def reference_loop(tracker, b, start, end, dead_cutoff, print_on_dead_loss, outputs):
    """ltt_run_beam_mode turn by turn, as lt_tracking_mod.f90:1612-1717."""
    n_tot = b.vec6.shape[1]
    n_print = max(1, _nint(print_on_dead_loss * n_tot))
    n_live_old = n_tot
    reports = []

    def emit(t):
        for every, cb in outputs:
            if every > 0 and t % every == 0:
                cb(t, b)

    if start == 0:
        emit(0)
    n_live = int(np.sum(b.state == L.ALIVE))
    for t in range(start, end):
        tracker.track_turns(b, 1, turn0=t)
        n_live = int(np.sum(b.state == L.ALIVE))
        if n_live_old - n_live >= n_print:
            reports.append((t + 1, n_tot - n_live))
            n_live_old = n_live
        if n_live == 0:
            return t + 1, "no_live_particles", n_live, reports
        if n_tot - n_live >= _nint(dead_cutoff * n_tot):
            return t + 1, "dead_cutoff", n_live, reports
        emit(t + 1)
    return end, "end_turn", n_live, reports


@pytest.fixture(scope="module")
def setup(oracle_lib):
    lat = rings.fodo_ring(apertures=True)
    # losses spread over the turns: 35 in the first turn, 47 after 3, 50 after 13, 54 after 30
    v0 = rings.gaussian_beam(rings.BeamSpec(300, 2e-6, 1e-6, 3e-3, 1e-2, seed=77))
    return lat, v0, oracle_lib


@pytest.mark.parametrize("dead_cutoff,print_loss,every,max_call,calls", [
    (1.0, -1.0, (5,), None, 6),          # no stop: outputs every 5 turns, six segments
    (50 / 300, 0.01, (4, 7), None, 6),   # five segments; the stop at 13 inside [12, 14): tracked again
    (50 / 300, 0.01, (), 3, 6),          # segments of 3 turns, the stop at 13 inside [12, 15)
    (0.02, -1.0, (1,), None, 1),         # a segment per turn, the stop after the first
])
def test_segmented_loop_equals_turn_by_turn(setup, dead_cutoff, print_loss, every, max_call, calls):
    lat, v0, lib = setup
    logs = {"seg": [], "ref": []}

    def outputs(tag):
        return [(e, (lambda e_: (lambda t, b: logs[tag].append((e_, t, int(np.sum(b.state == 1))))))(e))
                for e in every]

    b1 = Bunch.from_vec(v0.copy(), lat.p0c, lat.species.mass)
    b2 = Bunch.from_vec(v0.copy(), lat.p0c, lat.species.mass)
    tr1, tr2 = OracleTracker(lat, lib), OracleTracker(lat, lib)
    r = ltt.run_beam_mode(tr1, b1, 0, 30, dead_cutoff, print_loss, outputs("seg"), max_turns_per_call=max_call)
    t_ref, stop_ref, n_live_ref, reports_ref = reference_loop(tr2, b2, 0, 30, dead_cutoff, print_loss,
                                                              outputs("ref"))
    assert (r.ix_turn, r.stop, r.n_live) == (t_ref, stop_ref, n_live_ref)
    assert r.dead_reports == reports_ref
    assert logs["seg"] == logs["ref"]
    for a, c in ((b1.vec6, b2.vec6), (b1.state, b2.state), (b1.ix_ele_lost, b2.ix_ele_lost),
                 (b1.ix_turn_lost, b2.ix_turn_lost), (b1.beta, b2.beta)):
        assert np.array_equal(a, c)
    assert tr1.calls == calls


def test_stop_when_no_particle_is_left(setup):
    lat, v0, lib = setup
    b = Bunch.from_vec(v0.copy() * 30, lat.p0c, lat.species.mass)  # every particle hits an aperture
    r = ltt.run_beam_mode(OracleTracker(lat, lib), b, 0, 20)
    assert r.stop == "no_live_particles" and r.n_live == 0 and r.ix_turn == 1


def test_resumed_start_turn_has_no_start_output(setup):
    lat, v0, lib = setup
    seen = []
    b = Bunch.from_vec(v0.copy() * 0.1, lat.p0c, lat.species.mass)
    r = ltt.run_beam_mode(OracleTracker(lat, lib), b, 10, 16, outputs=[(2, lambda t, b_: seen.append(t))])
    assert seen == [12, 14, 16] and r.ix_turn == 16 and r.stop == "end_turn"


def reference_single(tracker, lat, vec, start, stop, every, only_last, averages):
    """ltt_run_single_mode for one particle, turn by turn
    (lt_tracking_mod.f90:1394-1450)."""
    b = Bunch.from_vec(vec.reshape(6, 1).copy(), lat.p0c, lat.species.mass)
    rows = [(start, b.vec6[:, 0].copy())]
    avg, sig, n_sum = np.zeros(6), np.zeros((6, 6)), 0
    n_turns = stop - start
    t_end = start
    for t in range(start, stop):
        tracker.track_turns(b, 1, turn0=t)
        t_end = t + 1
        if b.state[0] != L.ALIVE:
            break
        do_write = only_last < 1 or n_turns - t > only_last
        if every > 0 and do_write and (t + 1) % every == 0:
            rows.append((t + 1, b.vec6[:, 0].copy()))
        if averages:
            avg = avg + b.vec6[:, 0]
            sig = sig + np.outer(b.vec6[:, 0], b.vec6[:, 0])
            n_sum += 1
    if averages and n_sum:
        avg = avg / n_sum
        sig = sig / n_sum - np.outer(avg, avg)
    return t_end, rows, n_sum, avg, sig, b


@pytest.mark.parametrize("every,only_last,averages", [(3, -1, False), (1, 5, True), (0, -1, True), (4, -1, True)])
def test_single_mode_equals_one_particle_at_a_time(setup, every, only_last, averages):
    lat, v0, lib = setup
    idx = np.arange(0, 300, 15)  # 20 particles, several lost over the 20 turns
    v = v0[:, idx].copy()
    b = Bunch.from_vec(v.copy(), lat.p0c, lat.species.mass)
    r = ltt.run_single_mode(OracleTracker(lat, lib), b, 2, 22, every, only_last, averages=averages)
    n_lost = 0
    for k in range(v.shape[1]):
        t_end, rows, n_sum, avg, sig, bk = reference_single(OracleTracker(lat, lib), lat, v[:, k], 2, 22, every,
                                                             only_last, averages)
        n_lost += int(bk.state[0] != L.ALIVE)
        assert r.ix_turn[k] == t_end
        mine = [(t, vec) for t, i, vec in r.rows if i == k]
        assert [t for t, _ in mine] == [t for t, _ in rows]
        assert all(np.array_equal(a, c) for (_, a), (_, c) in zip(mine, rows))
        assert np.array_equal(b.vec6[:, k], bk.vec6[:, 0]) and b.state[k] == bk.state[0]
        if averages:
            assert r.n_sum[k] == n_sum
            assert np.array_equal(r.average[k], avg) and np.array_equal(r.sigma[k], sig)
    assert 0 < n_lost < v.shape[1]
