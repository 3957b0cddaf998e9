"""The synthetic rings and beams the benchmarks are defined on.

Ring (all configurations): 64 identical FODO cells plus one RF cavity and the
end marker, circumference 448.5 m, e- at 5 GeV, all elements bmad_standard:

    QF quadrupole L=0.4 k1=+0.8 | drift 0.3 | SF sextupole L=0.2 | drift 0.3 |
    sbend L=2.0 angle=2pi/128   | drift 0.3 | QD quadrupole L=0.4 k1=-0.8 |
    drift 0.3 | SD sextupole L=0.2 | drift 0.3 | sbend | drift 0.3

    rfcavity L=0.5, 5 MV, harmonic 748, phi0 at the stable zero crossing.

SF/SD k2 are fitted so both linear chromaticities are +1
(:func:`bgt.optics.fit_chromaticity`); the fitted values are stored below.

Workloads (particle counts, turns, errors) are documented with each builder.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import lattice as L

E_TOT = 5e9
N_CELL = 64
HARMONIC = 748
RF_VOLTAGE = 5e6
ANGLE = L.TWOPI / 128

# Fitted sextupole strengths (chromaticity +1 in both planes) and the
# matched optics at the start of the ring.  Produced by
# bgt.rings.fit_ring_optics() with the GPU tracker; reproduced on CPU by the
# test suite.
K2_SF = 3.51108791627275
K2_SD = -5.132216700784618
# stable zero crossing of the RF for this (above-transition) electron ring
PHI0 = 0.0


def p0c() -> float:
    return L.p0c_from_e_tot(E_TOT, L.M_ELECTRON)


def fodo_ring(k2_sf: Optional[float] = None, k2_sd: Optional[float] = None, apertures: bool = False,
              rf_on: bool = True, phi0: Optional[float] = None, name: str = "fodo64") -> L.Lattice:
    """Build the ring.  apertures=True adds config-1's apertures: elliptical
    20 mm x 10 mm half-axes on every quadrupole, rectangular 30 mm x 15 mm at
    the RF cavity."""
    k2_sf = K2_SF if k2_sf is None else k2_sf
    k2_sd = K2_SD if k2_sd is None else k2_sd
    phi0 = PHI0 if phi0 is None else phi0
    els: List[L.Element] = []

    def quad(nm, k1):
        e = L.Element("quadrupole", nm, {"l": 0.4, "k1": k1})
        if apertures:
            e.aperture_type = "elliptical"
            e.values.update(x1_limit=0.02, x2_limit=0.02, y1_limit=0.01, y2_limit=0.01)
        return e

    def drift(nm):
        return L.Element("drift", nm, {"l": 0.3})

    def sext(nm, k2):
        return L.Element("sextupole", nm, {"l": 0.2, "k2": k2})

    def bend(nm):
        return L.Element("sbend", nm, {"l": 2.0, "g": ANGLE / 2.0})

    for c in range(N_CELL):
        els += [quad(f"QF{c}", 0.8), drift(f"D1_{c}"), sext(f"SF{c}", k2_sf), drift(f"D2_{c}"), bend(f"BA{c}"),
                drift(f"D3_{c}"), quad(f"QD{c}", -0.8), drift(f"D4_{c}"), sext(f"SD{c}", k2_sd), drift(f"D5_{c}"),
                bend(f"BB{c}"), drift(f"D6_{c}")]
    circ = sum(e.v("l") for e in els) + 0.5
    pc = p0c()
    beta0 = pc / E_TOT
    rf = L.Element("rfcavity", "RF", {"l": 0.5, "voltage": RF_VOLTAGE if rf_on else 0.0, "phi0": phi0,
                                      "rf_frequency": HARMONIC * beta0 * L.C_LIGHT / circ})
    if apertures:
        rf.values.update(x1_limit=0.03, x2_limit=0.03, y1_limit=0.015, y2_limit=0.015)
    els.append(rf)
    els.append(L.Element("marker", "END"))
    lat = L.Lattice(els, L.Species("electron", L.M_ELECTRON, -1), pc, E_TOT, name)
    return lat.finalize()


@dataclass
class BeamSpec:
    n: int
    emit_x: float
    emit_y: float
    sigma_z: float
    sigma_pz: float
    seed: int


# config 0: 10k particles, 1000 turns, no apertures
CONFIG0_BEAM = BeamSpec(10_000, 1e-9, 10e-12, 3e-3, 1e-3, seed=20260001)
# config 1: 1M particles, 3x the config-0 emittances (sqrt(3) on each
# longitudinal sigma), 10k turns, apertures
CONFIG1_BEAM = BeamSpec(1_000_000, 3e-9, 30e-12, 3e-3 * math.sqrt(3), 1e-3 * math.sqrt(3), seed=20260002)

# Matched optics at the ring start (from fit_ring_optics); filled in below.
TWISS0 = dict(beta_a=11.887244599751257, alpha_a=-1.8074579900510381, beta_b=3.7441933691886216,
              alpha_b=0.47324178195194055, eta_x=0.7913233223685988, etap_x=0.127872130259893)
TUNES0 = (0.6749893337304752, 0.591269476707743)


def gaussian_beam(spec: BeamSpec, twiss: Optional[dict] = None, n: Optional[int] = None) -> np.ndarray:
    """Seeded 6D Gaussian (numpy Philox) matched to the periodic Twiss at the
    start: x = sqrt(eps*beta) u0 + eta*pz, px = sqrt(eps/beta)(u1 - alpha u0)
    + etap*pz, likewise y; z, pz independent.  Returns vec6 (6, n)."""
    tw = TWISS0 if twiss is None else twiss
    n = spec.n if n is None else n
    rng = np.random.Generator(np.random.Philox(spec.seed))
    u = rng.standard_normal((6, n))
    v = np.zeros((6, n))
    pz = spec.sigma_pz * u[5]
    v[5] = pz
    v[4] = spec.sigma_z * u[4]
    sx, sy = math.sqrt(spec.emit_x * tw["beta_a"]), math.sqrt(spec.emit_y * tw["beta_b"])
    v[0] = sx * u[0] + tw["eta_x"] * pz
    v[1] = math.sqrt(spec.emit_x / tw["beta_a"]) * (u[1] - tw["alpha_a"] * u[0]) + tw["etap_x"] * pz
    v[2] = sy * u[2]
    v[3] = math.sqrt(spec.emit_y / tw["beta_b"]) * (u[3] - tw["alpha_b"] * u[2])
    return v


def _trunc_gauss(rng, sigma, size):
    """Gaussian truncated at 3 sigma (resampled)."""
    x = rng.standard_normal(size)
    bad = np.abs(x) > 3
    while np.any(bad):
        x[bad] = rng.standard_normal(int(bad.sum()))
        bad = np.abs(x) > 3
    return sigma * x


def error_variants(n_variants: int, seed: int = 20260003, base: Optional[L.Lattice] = None,
                   apertures: bool = True) -> List[L.Lattice]:
    """Config 2: variants of the config-1 ring.  Every quadrupole and
    sextupole gets, per variant, Gaussian errors truncated at 3 sigma:
    x/y offsets sigma 50 um, roll (tilt) sigma 100 urad, and relative normal
    and skew multipoles of Bmad orders n = 3..6 with sigma 1e-4 at
    r0_mag = 10 mm (scaled by the element's main strength, Bmad's
    scale_multipoles convention)."""
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for v in range(n_variants):
        lat = fodo_ring(apertures=apertures, name=f"fodo64_err{v}")
        for e in lat.elements:
            if e.key not in ("quadrupole", "sextupole"):
                continue
            e.values["x_offset"] = float(_trunc_gauss(rng, 50e-6, 1)[0])
            e.values["y_offset"] = float(_trunc_gauss(rng, 50e-6, 1)[0])
            e.values["tilt"] = float(_trunc_gauss(rng, 100e-6, 1)[0])
            e.values["r0_mag"] = 0.01
            an = _trunc_gauss(rng, 1e-4, 4)
            bn = _trunc_gauss(rng, 1e-4, 4)
            for k, n in enumerate(range(3, 7)):
                e.a_pole[n] = float(an[k])
                e.b_pole[n] = float(bn[k])
            e.num_steps = 0
            e.values.pop("ds_step", None)
        out.append(lat.finalize())
    return out


def sextupole_variants(n_variants: int, seed: int = 20260004, spread: float = 0.30,
                       apertures: bool = True) -> List[L.Lattice]:
    """Config 4: variants with SF/SD k2 drawn uniformly at +/-spread around
    the fitted values, no other errors."""
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    for v in range(n_variants):
        f = 1 + rng.uniform(-spread, spread, 2)
        out.append(fodo_ring(K2_SF * f[0], K2_SD * f[1], apertures=apertures, name=f"fodo64_sx{v}"))
    return out


@dataclass
class DAGrid:
    n_angle: int
    n_radius: int
    r_max: float
    deltas: Sequence[float]
    n_turns: int
    angle_min: float = 0.0
    angle_max: float = math.pi


# config 2: 40 angles x 64 radii (0-25 mm in x), delta in {-1%, 0, +1%}, 20k turns
CONFIG2_GRID = DAGrid(40, 64, 0.025, (-0.01, 0.0, 0.01), 20_000)
# config 4: 32 angles x 64 radii, delta = 0, 20k turns
CONFIG4_GRID = DAGrid(32, 64, 0.025, (0.0,), 20_000)
