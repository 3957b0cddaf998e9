"""long_term_tracking's BEAM-mode and single-particle turn loops on the tracker.

Restates ``ltt_run_beam_mode`` (bsim/modules/lt_tracking_mod.f90:1571-1719)
for one bunch: the outputs at the start turn, the per-turn bookkeeping of
live particles, the "cumulative number dead" reports every
``print_on_dead_loss`` of the bunch, the stop when no particle is left or
when the losses reach ``dead_cutoff`` of the bunch, and the outputs after
every turn -- here callbacks, each with its own turn interval, as the
reference's averages / beam / per-particle writers each test their own
``*_every_n_turns``.

The tracker runs many turns per call, so the loop tracks in segments that
end at the next turn with an output and replays the per-turn decisions from
the particles' loss turns afterwards.  When a stop falls inside a segment
the segment is tracked again from its start, as far as the stop turn only:
tracking is deterministic, so the bunch then holds exactly the state the
turn-by-turn loop stops with.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

from . import lattice as L


def _nint(x: float) -> int:
    """Fortran nint: round half away from zero."""
    return int(math.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)


@dataclass
class BeamModeResult:
    ix_turn: int  # the turn index after the last turn tracked (bunch%ix_turn)
    stop: str  # "end_turn", "no_live_particles" or "dead_cutoff"
    n_live: int
    dead_reports: List[Tuple[int, int]] = field(default_factory=list)  # (turn, cumulative dead)


def run_beam_mode(tracker, bunch, ix_start_turn: int, ix_end_turn: int, dead_cutoff: float = 1.0,
                  print_on_dead_loss: float = -1.0,
                  outputs: Sequence[Tuple[int, Callable[[int, object], None]]] = (),
                  max_turns_per_call: Optional[int] = None) -> BeamModeResult:
    """Track `bunch` from turn `ix_start_turn` to `ix_end_turn` with
    `tracker` (anything with ``track_turns(bunch, n_turns, turn0=)``, such as
    :class:`bgt.track.Tracker`).  `outputs` holds (every, callback) pairs:
    callback(turn, bunch) runs at the start turn when it is 0 and after every
    turn that is a multiple of `every` (every <= 0: never)."""
    n_tot = bunch.vec6.shape[1]
    n_print = max(1, _nint(print_on_dead_loss * n_tot))
    n_cut = _nint(dead_cutoff * n_tot)
    n_live_old = n_tot
    res = BeamModeResult(ix_start_turn, "end_turn", int(np.sum(bunch.state == L.ALIVE)))

    def emit(turn: int):
        for every, cb in outputs:
            if every > 0 and turn % every == 0:
                cb(turn, bunch)

    if ix_start_turn == 0:
        emit(0)
    turn = ix_start_turn
    while turn < ix_end_turn:
        stop_at = ix_end_turn
        for every, _ in outputs:
            if every > 0:
                stop_at = min(stop_at, (turn // every + 1) * every)
        if max_turns_per_call:
            stop_at = min(stop_at, turn + max_turns_per_call)
        saved = (bunch.vec6.copy(), bunch.beta.copy(), bunch.state.copy(), bunch.ix_ele_lost.copy(),
                 bunch.ix_turn_lost.copy())
        alive0 = bunch.state == L.ALIVE
        tracker.track_turns(bunch, stop_at - turn, turn0=turn)
        # live count after each turn of the segment, from the loss turns
        lost_turn = np.where(alive0 & (bunch.state != L.ALIVE), bunch.ix_turn_lost, -1)
        stop_turn, reason = None, None
        for t in range(turn, stop_at):
            n_live = int(np.sum(alive0)) - int(np.sum((lost_turn >= 0) & (lost_turn <= t)))
            if n_live_old - n_live >= n_print:
                res.dead_reports.append((t + 1, n_tot - n_live))
                n_live_old = n_live
            if n_live == 0:
                stop_turn, reason = t + 1, "no_live_particles"
                break
            if n_tot - n_live >= n_cut:
                stop_turn, reason = t + 1, "dead_cutoff"
                break
            res.n_live = n_live
        if stop_turn is not None:
            if stop_turn < stop_at:
                # track the segment again, up to the stop turn only
                (bunch.vec6[:], bunch.beta[:], bunch.state[:], bunch.ix_ele_lost[:],
                 bunch.ix_turn_lost[:]) = saved
                tracker.track_turns(bunch, stop_turn - turn, turn0=turn)
            res.ix_turn = stop_turn
            res.stop = reason
            res.n_live = int(np.sum(bunch.state == L.ALIVE))
            return res
        turn = stop_at
        res.ix_turn = turn
        emit(turn)
    return res


@dataclass
class SingleModeResult:
    ix_turn: np.ndarray  # per particle: the turn after its last tracked turn (the loss turn + 1 when lost)
    rows: List[Tuple[int, int, np.ndarray]]  # (turn, particle, vec6) phase-space output rows
    n_sum: np.ndarray  # per particle: turns summed into the averages
    average: Optional[np.ndarray] = None  # [n, 6]: mean of vec over the summed turns
    sigma: Optional[np.ndarray] = None  # [n, 6, 6]: <vec vec^T> - average average^T


def run_single_mode(tracker, bunch, ix_turn_start: int, ix_turn_stop: int, particle_output_every_n_turns: int = 0,
                    output_only_last_turns: int = -1, n_turns: Optional[int] = None,
                    averages: bool = False) -> SingleModeResult:
    """The single-particle turn loop ``ltt_run_single_mode``
    (bsim/modules/lt_tracking_mod.f90:1333-1465) for every particle of
    `bunch` at once -- the particles are independent, so one call per turn
    (or per output interval) tracks them all, each stopping at its own loss.
    Per particle: an output row at the start turn and after every turn that
    is a multiple of `particle_output_every_n_turns` (while ``n_turns -
    i_turn > output_only_last_turns`` or that bound is below 1, as the
    reference tests it), nothing after the particle is lost; with `averages`
    the mean and the second moments of vec over the turns survived
    (ltt_write_single_mode_sigma_file, :2714-2749)."""
    n = bunch.vec6.shape[1]
    n_turns = (ix_turn_stop - ix_turn_start) if n_turns is None else n_turns
    every = particle_output_every_n_turns
    res = SingleModeResult(np.full(n, ix_turn_start, np.int64), [], np.zeros(n, np.int64))
    acc = np.zeros((n, 6)) if averages else None
    acc2 = np.zeros((n, 6, 6)) if averages else None
    alive = bunch.state == L.ALIVE
    for i in np.nonzero(alive)[0]:
        res.rows.append((ix_turn_start, int(i), bunch.vec6[:, i].copy()))
    turn = ix_turn_start
    while turn < ix_turn_stop and np.any(bunch.state == L.ALIVE):
        # without averages only the output turns need the coordinates
        stop_at = turn + 1
        if not averages:
            stop_at = ix_turn_stop
            if every > 0:
                stop_at = min(stop_at, (turn // every + 1) * every)
        alive0 = bunch.state == L.ALIVE
        tracker.track_turns(bunch, stop_at - turn, turn0=turn)
        alive1 = bunch.state == L.ALIVE
        lost = alive0 & ~alive1
        res.ix_turn[lost] = bunch.ix_turn_lost[lost] + 1
        res.ix_turn[alive1] = stop_at
        t = stop_at - 1  # the last turn of the segment
        if averages:
            v = bunch.vec6[:, alive1].T
            acc[alive1] += v
            acc2[alive1] += v[:, :, None] * v[:, None, :]
            res.n_sum[alive1] += 1
        do_write = output_only_last_turns < 1 or n_turns - t > output_only_last_turns
        if every > 0 and do_write and (t + 1) % every == 0:
            for i in np.nonzero(alive1)[0]:
                res.rows.append((t + 1, int(i), bunch.vec6[:, i].copy()))
        turn = stop_at
    if averages:
        ok = res.n_sum > 0
        res.average = np.zeros((n, 6))
        res.sigma = np.zeros((n, 6, 6))
        res.average[ok] = acc[ok] / res.n_sum[ok, None]
        res.sigma[ok] = acc2[ok] / res.n_sum[ok, None, None] - \
            res.average[ok][:, :, None] * res.average[ok][:, None, :]
    return res
