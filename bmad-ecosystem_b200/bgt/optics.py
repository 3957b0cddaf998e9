"""Linear optics around a one-turn map: closed orbit, one-turn matrix, Twiss,
tunes and chromaticity.  The map is any callable taking a (6, n) float64
array of coordinates and returning them after one turn -- in the product the
GPU tracker (:class:`bgt.track.Tracker`).

Restates the host-side setup the reference does before tracking:
closed orbit (``bmad/code/closed_orbit_calc.f90:81``), one-turn matrix and
Twiss (``bmad/code/twiss_at_start.f90:29``), and the chromaticity fit of
``bmad/code/chrom_tune.f90:29`` (here a Newton fit of the two sextupole
families to a target chromaticity).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

OneTurn = Callable[[np.ndarray], np.ndarray]


def closed_orbit(one_turn: OneTurn, delta: float = 0.0, six_d: bool = False, guess=None, tol: float = 1e-14,
                 max_iter: int = 20, h: float = 1e-9) -> np.ndarray:
    """Newton iteration on x -> M(x) - x.  4D mode keeps pz = delta fixed and
    ignores z; 6D mode solves all six coordinates (RF on)."""
    co = np.zeros(6) if guess is None else np.array(guess, dtype=np.float64)
    if not six_d:
        co[5] = delta
    idx = list(range(6)) if six_d else [0, 1, 2, 3]
    for _ in range(max_iter):
        pts = np.repeat(co[:, None], 1 + len(idx), axis=1)
        for j, k in enumerate(idx):
            pts[k, 1 + j] += h
        out = one_turn(pts.copy())
        f0 = out[:, 0] - pts[:, 0]
        jac = np.zeros((len(idx), len(idx)))
        for j in range(len(idx)):
            jac[:, j] = (out[idx, 1 + j] - out[idx, 0]) / h
        a = jac - np.eye(len(idx))
        step = np.linalg.solve(a, -f0[idx])
        co[idx] = co[idx] + step
        if np.max(np.abs(step)) < tol:
            break
    return co


def one_turn_matrix(one_turn: OneTurn, orbit: np.ndarray, h: float = 1e-6) -> np.ndarray:
    """Central-difference 6x6 Jacobian of the one-turn map at `orbit`."""
    pts = np.repeat(orbit[:, None], 12, axis=1)
    for k in range(6):
        pts[k, 2 * k] += h
        pts[k, 2 * k + 1] -= h
    out = one_turn(pts.copy())
    m = np.zeros((6, 6))
    for k in range(6):
        m[:, k] = (out[:, 2 * k] - out[:, 2 * k + 1]) / (2 * h)
    return m


@dataclass
class Twiss:
    beta_a: float
    alpha_a: float
    beta_b: float
    alpha_b: float
    eta_x: float
    etap_x: float
    eta_y: float
    etap_y: float
    tune_a: float
    tune_b: float


def _plane(m2: np.ndarray):
    c = 0.5 * (m2[0, 0] + m2[1, 1])
    if abs(c) >= 1:
        raise ValueError("unstable plane (|cos mu| >= 1)")
    mu = math.acos(c)
    if m2[0, 1] < 0:
        mu = 2 * math.pi - mu
    s = math.sin(mu)
    beta = m2[0, 1] / s
    alpha = (m2[0, 0] - m2[1, 1]) / (2 * s)
    return beta, alpha, mu / (2 * math.pi)


def twiss(one_turn_4d: OneTurn, delta: float = 0.0) -> Twiss:
    """Twiss at the start from the 4D map (pz fixed, RF off or ignored)."""
    co = closed_orbit(one_turn_4d, delta=delta)
    m = one_turn_matrix(one_turn_4d, co)
    ba, aa, qa = _plane(m[0:2, 0:2])
    bb, ab, qb = _plane(m[2:4, 2:4])
    # periodic dispersion: (I - M4) eta = M4,delta
    m4 = m[0:4, 0:4]
    eta = np.linalg.solve(np.eye(4) - m4, m[0:4, 5])
    return Twiss(ba, aa, bb, ab, eta[0], eta[1], eta[2], eta[3], qa, qb)


def chromaticity(one_turn_4d: OneTurn, d_delta: float = 1e-4):
    """(xi_a, xi_b) = dQ/dpz by tunes at +/- d_delta (chrom_calc style)."""
    tp = twiss(one_turn_4d, +d_delta)
    tm = twiss(one_turn_4d, -d_delta)

    def dq(a, b):
        d = a - b
        if d > 0.5:
            d -= 1
        if d < -0.5:
            d += 1
        return d

    return dq(tp.tune_a, tm.tune_a) / (2 * d_delta), dq(tp.tune_b, tm.tune_b) / (2 * d_delta)


def fit_chromaticity(make_map: Callable[[float, float], OneTurn], k2_guess, target=(1.0, 1.0), tol=1e-10,
                     max_iter: int = 8, dk: float = 1e-3):
    """Newton fit of two sextupole strengths (k2_f, k2_d) so the
    chromaticities equal `target`.  make_map(k2_f, k2_d) returns a 4D
    one-turn map for those settings."""
    k = np.array(k2_guess, dtype=np.float64)
    tgt = np.array(target, dtype=np.float64)
    xi = np.array(chromaticity(make_map(*k)))
    for _ in range(max_iter):
        if np.max(np.abs(xi - tgt)) < tol:
            break
        jac = np.zeros((2, 2))
        for j in range(2):
            kk = k.copy()
            kk[j] += dk
            jac[:, j] = (np.array(chromaticity(make_map(*kk))) - xi) / dk
        k = k + np.linalg.solve(jac, tgt - xi)
        xi = np.array(chromaticity(make_map(*k)))
    return k, xi


def synchrotron_tune(one_turn_6d: OneTurn) -> Optional[float]:
    """Synchrotron tune from the 6D one-turn matrix (None if unstable)."""
    co = closed_orbit(one_turn_6d, six_d=True)
    m = one_turn_matrix(one_turn_6d, co)
    ev = np.linalg.eigvals(m)
    # the longitudinal pair is the one whose eigenvector lives in (z, pz);
    # take the eigenvalue pair with the smallest |arg|
    args = np.abs(np.angle(ev))
    mags = np.abs(ev)
    if np.max(np.abs(mags - 1)) > 1e-6:
        return None
    return float(np.min(args) / (2 * math.pi))
