"""Momentum aperture by tracking, every start location in one launch per
search step.

Restates bsim/aperture_by_tracking (aperture_by_tracking.f90:254-380 and
aperture_by_tracking_mod.f90:275-345): for each slice location s, a particle
starts on the closed orbit at s with its pz kicked by +delta (positive
aperture) or -delta (negative aperture), is tracked `n_turns` turns, and the
largest surviving |delta| is found by the program's bracketing binary search
(double / halve until the aperture is bracketed, then move half the bracket
towards the other side; stop when |high - low| / min(|high|, |low|) falls
below the target accuracy; |delta| > 1 or < 1e-6 ends the search).

GPU form: slice i is a lattice variant -- the ring rotated to start at the
slice's element, every element keeping its Bmad index -- so all slices and
both signs are one batch, and each search step is one launch over all
searches still running.  The search state (bracket flags, last high / low,
accuracy) is kept per search in arrays and advanced exactly as
binary_search does.
"""
from __future__ import annotations

import copy
from dataclasses import dataclass
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import lattice as L


def rotated(lat: L.Lattice, start: int) -> L.Lattice:
    """The ring starting at element position `start` (0-based); elements keep
    their Bmad index."""
    els = [copy.deepcopy(e) for e in lat.elements[start:] + lat.elements[:start]]
    ix = [e.ix_ele for e in els]
    out = L.Lattice(els, lat.species, lat.p0c, lat.e_tot, f"{lat.name}@{start}").finalize()
    for e, i in zip(out.elements, ix):
        e.ix_ele = i
    return out


@dataclass
class SearchState:
    """binary_search's saved variables, one entry per search."""
    delta: np.ndarray
    high_found: np.ndarray
    low_found: np.ndarray
    bracket: np.ndarray
    last_high: np.ndarray
    last_low: np.ndarray
    accuracy: np.ndarray

    @classmethod
    def start(cls, n: int, first_guess: float) -> "SearchState":
        z = np.zeros(n)
        f = np.zeros(n, bool)
        return cls(np.full(n, first_guess), f.copy(), f.copy(), f.copy(), z.copy(), z.copy(), np.full(n, 10.0))


def binary_search_step(s: SearchState, lost: np.ndarray, active: np.ndarray):
    """One call of binary_search(lost, delta_m, accuracy, .false.)
    (aperture_by_tracking_mod.f90:275-345) for the active searches."""
    a = active
    nb = a & ~s.bracket
    # not yet bracketed: halve after a loss (until a survivor is known),
    # double after a survivor (until a loss is known)
    hl = nb & lost
    s.high_found[hl] = True
    s.last_high[hl] = s.delta[hl]
    m = hl & ~s.low_found
    s.delta[m] = s.delta[m] / 2.0
    ls = nb & ~lost
    s.low_found[ls] = True
    s.last_low[ls] = s.delta[ls]
    m = ls & ~s.high_found
    s.delta[m] = s.delta[m] * 2.0
    s.bracket[nb] = s.high_found[nb] & s.low_found[nb]
    s.accuracy[nb] = 10.0
    # bracketed: move half the bracket
    br = a & s.bracket
    m = br & lost
    s.last_high[m] = s.delta[m]
    s.delta[m] = s.delta[m] - np.abs(s.delta[m] - s.last_low[m]) / 2.0
    m = br & ~lost
    s.last_low[m] = s.delta[m]
    s.delta[m] = s.delta[m] + np.abs(s.last_high[m] - s.delta[m]) / 2.0
    s.accuracy[br] = np.abs(s.last_high[br] - s.last_low[br]) / np.minimum(np.abs(s.last_high[br]),
                                                                           np.abs(s.last_low[br]))
    # extreme values end the search
    big = a & (np.abs(s.delta) > 1.0)
    s.accuracy[big] = 0.0
    s.last_high[big] = 1.1
    s.last_low[big] = 0.9
    small = a & (np.abs(s.delta) < 1.0e-6)
    s.accuracy[small] = 0.0
    s.last_high[small] = 2.0e-6
    s.last_low[small] = 0.0


# lost_fn(vec6[6, m], variant[m]) -> bool[m]: tracked n_turns from each
# variant's start, True when the particle did not survive
LostFn = Callable[[np.ndarray, np.ndarray], np.ndarray]


def search(lost_fn: LostFn, start_orbits: np.ndarray, first_guess: float = 0.001, target_accuracy: float = 0.01,
           signs: Sequence[int] = (1, -1), coord: int = 5, max_steps: int = 200):
    """Apertures [n_slices, len(signs)] (signed: sign * final delta) and the
    number of search steps."""
    ns = start_orbits.shape[0]
    nk = len(signs)
    n = ns * nk
    st = SearchState.start(n, first_guess)
    slice_of = np.repeat(np.arange(ns, dtype=np.int32), nk)
    sign_of = np.tile(np.array(signs, dtype=np.float64), ns)
    steps = 0
    while steps < max_steps:
        active = st.accuracy > target_accuracy
        if not active.any():
            break
        idx = np.nonzero(active)[0]  # slice-major: variant ids stay sorted
        v = start_orbits[slice_of[idx]].T.copy()
        v[coord] = v[coord] + sign_of[idx] * st.delta[idx]
        lost = np.zeros(n, bool)
        lost[idx] = lost_fn(np.ascontiguousarray(v), slice_of[idx])
        binary_search_step(st, lost, active)
        steps += 1
    ap = (sign_of * st.delta).reshape(ns, nk)
    return ap, steps


def closed_orbit_at(one_pass: Callable[[np.ndarray, int, int], np.ndarray], co0: np.ndarray,
                    starts: Sequence[int]) -> np.ndarray:
    """Closed orbit at each start element by tracking the orbit at element 0
    element by element (track_s_to_s, aperture_by_tracking.f90:254-256).
    one_pass(vec6[6, 1], e_begin, e_end) tracks through positions
    [e_begin, e_end)."""
    out = np.zeros((len(starts), 6))
    v = np.array(co0, dtype=np.float64).reshape(6, 1)
    pos = 0
    for k, s in enumerate(starts):
        if s > pos:
            v = one_pass(v, pos, s)
            pos = s
        out[k] = v[:, 0]
    return out


@dataclass
class MomentumAperture:
    starts: List[int]
    ix_ele: List[int]
    aperture: np.ndarray  # [n_slices, 2] (+, -)
    steps: int


def momentum_aperture(lat: L.Lattice, starts: Sequence[int], n_turns: int, first_guess: float = 0.001,
                      target_accuracy: float = 0.01, device: int = 0, tracker_cls=None) -> MomentumAperture:
    """GPU momentum aperture at the start of each element position in
    `starts` (ascending 0-based positions)."""
    from . import da
    from .track import Tracker

    tracker_cls = tracker_cls or Tracker
    base = tracker_cls(lat, device=device)
    co0 = da.variant_optics(da.tracker_one_turn(base), 1).closed_orbit[0]

    def one_pass(v, b, e):
        bb = base.make_bunch(v.copy())
        base.track_elements(bb, b, e)
        return bb.vec6

    sco = closed_orbit_at(one_pass, co0, starts)
    rings_ = tracker_cls([rotated(lat, s) for s in starts], device=device)

    def lost_fn(v6, var):
        b = rings_.make_bunch(v6)
        rings_.track_turns(b, n_turns, variant=var)
        return b.state != 1

    ap, steps = search(lost_fn, sco, first_guess, target_accuracy)
    return MomentumAperture(list(starts), [lat.elements[s].ix_ele for s in starts], ap, steps)
