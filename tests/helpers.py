"""Shared fixtures for parity tests: an element zoo, seeded particles, and
the oracle / GPU runners compared by the tests."""
from __future__ import annotations

import math

import numpy as np

from bgt import lattice as L
from bgt import rings

# Tolerances (FP64).  Per coordinate c, a GPU value g and oracle value o agree
# when |g - o| <= RTOL * (|o| + rms_c), rms_c the bunch RMS of coordinate c:
# relative to the value, with the coordinate's bunch scale as the floor for
# values that pass near zero.
RTOL_ONE_TURN = 1e-13
RTOL_1000_TURNS = 1e-9
# Against the C-library (glibc) build of the oracle, whole-ring results carry
# glibc's own rounding: glibc 2.39 is not correctly rounded on ~0.17% of asin
# and ~0.01-0.03% of sin/cos/atan2 arguments on this path, and the exact bend
# (px from phi_1 + angle - angle_p, ~5e-2 angles cancelling to ~1e-5) turns a
# one-ulp change into ~1e-12 relative.  The device is bit-identical to the
# correctly rounded oracle, and the correctly rounded and glibc oracles -- both
# on the CPU -- differ by exactly these amounts, so the floor below is the
# reference's own libm sensitivity, not a device error.
RTOL_LIBM_ONE_TURN = 1e-11


def rtol_vs_glibc_one_element(ele) -> float:
    """Bound of one element against the C-library oracle: RTOL_ONE_TURN,
    except for a bend with fringe_type full, whose exact (PTC) edge divides
    the difference of two asin values of the edge-angle size by g + dg
    (ptc_wedger, fringe_mod.f90:1020-1123): a one-ulp misrounding of glibc's
    asin moves z by ~1e-13 relative to the bunch size there, the
    reference's own sensitivity to its libm, bounded by RTOL_LIBM_ONE_TURN."""
    return RTOL_LIBM_ONE_TURN if (ele.key == "sbend" and ele.fringe_type == "full") else RTOL_ONE_TURN
RTOL_LIBM_1000_TURNS = 1e-7


def zoo_lattice(apertures: bool = True) -> L.Lattice:
    """One of every element form the GPU supports, at the 5 GeV ring energy,
    with misalignments, multipoles, edges and apertures."""
    E = []
    E.append(L.Element("drift", "D", {"l": 0.7}))
    E.append(L.Element("quadrupole", "Q0", {"l": 0.4, "k1": 0.8}))
    E.append(L.Element("quadrupole", "QERR", {"l": 0.4, "k1": -0.7, "x_offset": 2e-4, "y_offset": -1e-4,
                                              "tilt": 3e-3, "r0_mag": 0.01},
                       a_pole={3: 2e-4, 5: -1e-4}, b_pole={3: -3e-4, 4: 1e-4, 6: 2e-4}))
    E.append(L.Element("quadrupole", "QPITCH", {"l": 0.5, "k1": 0.6, "x_pitch": 2e-4, "y_pitch": -3e-4,
                                                "z_offset": 1e-3, "hkick": 1e-5}))
    E.append(L.Element("quadrupole", "QZERO", {"l": 0.3, "k1": 0.0, "hkick": 2e-5}))
    E.append(L.Element("sextupole", "S", {"l": 0.2, "k2": 25.0}))
    E.append(L.Element("sextupole", "SERR", {"l": 0.2, "k2": -30.0, "x_offset": 1e-4, "tilt": -2e-3,
                                             "r0_mag": 0.01}, a_pole={4: 1e-4}, b_pole={5: 2e-4}))
    E.append(L.Element("octupole", "O", {"l": 0.3, "k3": 300.0, "tilt": 0.1}, num_steps=4))
    E.append(L.Element("thick_multipole", "TM", {"l": 0.5, "x_offset": 1e-4}, a_pole={2: 1.0}, b_pole={3: 20.0}))
    E.append(L.Element("sbend", "B", {"l": 2.0, "g": rings.ANGLE / 2.0}))
    E.append(L.Element("sbend", "BE", {"l": 1.5, "g": 0.02, "e1": 0.05, "e2": -0.03, "fint": 0.5, "hgap": 0.02}))
    E.append(L.Element("sbend", "BK1", {"l": 1.2, "g": 0.015, "k1": 0.2, "e1": 0.02, "e2": 0.01}))
    E.append(L.Element("sbend", "BMUL", {"l": 1.0, "g": 0.03, "k2": 2.0, "ref_tilt": 0.05}, b_pole={4: 1e-3}))
    E.append(L.Element("sbend", "BHARD", {"l": 1.0, "g": -0.01, "e1": 0.1, "e2": 0.1, "fint": 0.3, "hgap": 0.05},
                       fringe_type="hard_edge_only"))
    E.append(L.Element("multipole", "M", {"x_offset": 1e-4}, a_pole={1: 0.05, 3: 40.0}, b_pole={1: 0.2, 3: 0.7}))
    E.append(L.Element("multipole", "M0", {}, a_pole={0: 1e-4, 2: 3.0}))
    E.append(L.Element("ab_multipole", "AB", {"x_offset": 2e-4, "tilt": 0.1}, a_pole={2: 1.0}, b_pole={2: 2.0}))
    E.append(L.Element("hkicker", "HK", {"l": 0.2, "kick": 1e-5}))
    E.append(L.Element("vkicker", "VK", {"l": 0.2, "kick": -2e-5}))
    E.append(L.Element("kicker", "K", {"l": 0.3, "hkick": 1e-5, "vkick": 2e-5}))
    E.append(L.Element("monitor", "MON", {"l": 0.1}))
    E.append(L.Element("instrument", "INS", {"l": 0.1, "x_offset": 1e-4}))
    E.append(L.Element("rcollimator", "RC", {"l": 0.2, "x1_limit": 0.02, "x2_limit": 0.02, "y1_limit": 0.01,
                                             "y2_limit": 0.012}))
    E.append(L.Element("ecollimator", "EC", {"l": 0.2, "x1_limit": 0.015, "x2_limit": 0.02, "y1_limit": 0.01,
                                             "y2_limit": 0.01}))
    E.append(L.Element("rfcavity", "RF", {"l": 0.5, "voltage": 5e6, "phi0": 0.02, "rf_frequency": 499.98e6}))
    E.append(L.Element("rfcavity", "RFMIS", {"l": 0.6, "voltage": 2e6, "phi0": -0.1, "rf_frequency": 499.98e6,
                                             "x_offset": 1e-4, "y_pitch": 1e-4, "tilt": 0.05}, num_steps=7))
    E.append(L.Element("marker", "MK"))
    E.append(L.Element("quadrupole", "QOFF", {"l": 0.4, "k1": 1.0}, is_on=False))
    E.append(L.Element("sextupole", "SOFF", {"l": 0.2, "k2": 50.0}, is_on=False))
    if apertures:
        E[1].aperture_type = "elliptical"
        E[1].values.update(x1_limit=0.02, x2_limit=0.02, y1_limit=0.01, y2_limit=0.01)
        E[5].values.update(x1_limit=0.025, x2_limit=0.02, y1_limit=0.0, y2_limit=0.012)
        E[5].aperture_at = "both_ends"
        E[-3].aperture_type = "elliptical"
        E[-3].values.update(x1_limit=0.01, x2_limit=0.012, y1_limit=0.008, y2_limit=0.008)
    lat = L.Lattice(E, L.Species("electron", L.M_ELECTRON, -1), rings.p0c(), rings.E_TOT, "zoo")
    return lat.finalize()


def rare_zoo_lattice() -> L.Lattice:
    """Element forms that only the device's RARE kernels handle: misaligned
    bends (offset_particle's bend geometry, with g, ref_tilt or roll), the
    straight geometry of a misaligned g = 0 bend, electric multipoles in bends
    and quadrupoles, the hard-edge multipole fringe, the soft-edge quadrupole
    fringe, the SAD soft and linear bend edges, an RF coupler kick, a
    misaligned collimator whose aperture moves with it and the exact bend
    edge of fringe_type full (with g + dg = 0 too) -- at the 5 GeV ring
    energy."""
    E = []
    E.append(L.Element("drift", "D", {"l": 0.5}))
    E.append(L.Element("sbend", "BMIS", {"l": 1.0, "g": 0.02, "e1": 0.03, "e2": 0.01, "x_offset": 1e-4,
                                         "y_offset": -2e-4, "z_offset": 1e-3, "x_pitch": 1e-4, "y_pitch": -2e-4,
                                         "ref_tilt": 0.05}))
    E.append(L.Element("sbend", "BROLL", {"l": 1.5, "g": 0.015, "roll": 2e-3, "x_offset": 1e-4}))
    E.append(L.Element("sbend", "BSTRAIGHT", {"l": 0.8, "k1": 0.1, "x_offset": 1e-4, "y_pitch": 1e-4}))
    E.append(L.Element("sbend", "BG0TILT", {"l": 0.8, "k1": 0.15, "ref_tilt": 0.1, "y_offset": 1e-4}))
    E.append(L.Element("sbend", "BELEC", {"l": 1.0, "g": 0.01, "e1": 0.05}, b_pole_elec={0: 2e4, 1: 5e6},
                       a_pole_elec={2: 1e8}))
    E.append(L.Element("sbend", "BELECMIS", {"l": 0.6, "g": 0.01, "e1": 0.1, "e2": 0.2, "x_offset": 2e-4,
                                             "y_pitch": 1e-4, "ref_tilt": 0.1, "vkick": -1e-5, "r0_mag": 2.0,
                                             "r0_elec": 3.0}, num_steps=10,
                       a_pole={0: 1e-4, 1: 1e-3}, a_pole_elec={1: 2e6}, b_pole_elec={0: -2e5}))
    E.append(L.Element("quadrupole", "QELEC", {"l": 0.4, "k1": 0.7, "x_offset": 1e-4, "tilt": 0.01},
                       num_steps=4, fringe_type="full", a_pole_elec={1: 3e6}, b_pole_elec={0: 1e5}))
    E.append(L.Element("sextupole", "SHARD", {"l": 0.2, "k2": 30.0}, fringe_type="hard_edge_only"))
    E.append(L.Element("quadrupole", "QSOFT", {"l": 0.4, "k1": 0.9, "fq1": 2e-3, "fq2": 1e-3}, fringe_type="full"))
    E.append(L.Element("sbend", "BSOFT", {"l": 1.0, "g": 0.02, "e1": 0.05, "e2": 0.02, "fint": 0.5, "hgap": 0.03},
                       fringe_type="soft_edge_only"))
    E.append(L.Element("sbend", "BSAD", {"l": 1.0, "g": -0.015, "e1": 0.08, "fint": 0.4, "hgap": 0.02},
                       fringe_type="sad_full"))
    E.append(L.Element("sbend", "BLIN", {"l": 0.8, "g": 0.01, "e1": 0.1, "e2": -0.05, "fint": 0.3, "hgap": 0.02},
                       fringe_type="linear_edge"))
    E.append(L.Element("quadrupole", "QSOFT2", {"l": 0.3, "k1": -1.2, "fq1": 0.05, "fq2": 0.02},
                       fringe_type="soft_edge_only"))
    E.append(L.Element("rfcavity", "RFCPL", {"l": 0.6, "voltage": 2e6, "phi0": 0.05, "rf_frequency": 499.98e6,
                                             "coupler_strength": 0.05, "coupler_angle": 0.1, "coupler_phase": 0.02},
                       num_steps=6, coupler_at="both_ends"))
    E.append(L.Element("ecollimator", "ECMIS", {"l": 0.2, "x1_limit": 0.015, "x2_limit": 0.0165, "y1_limit": 0.01,
                                                "y2_limit": 0.01, "x_offset": 5e-4, "tilt": 0.2}))
    # fringe_type full: the exact (PTC) bend edge inside the k1 hard-edge fringe
    E.append(L.Element("sbend", "BFULL", {"l": 1.0, "g": 0.02, "k1": 0.05, "e1": 0.06, "e2": 0.03, "fint": 0.5,
                                          "hgap": 0.03}, fringe_type="full"))
    E.append(L.Element("sbend", "BFULLMIS", {"l": 0.6, "g": 0.01, "e1": 0.1, "e2": 0.2, "fint": 0.7, "hgap": 0.05,
                                             "x_offset": 2e-4, "y_pitch": 1e-4, "ref_tilt": 0.1, "vkick": -1e-5,
                                             "r0_mag": 2.0, "r0_elec": 3.0}, num_steps=10, fringe_type="full",
                       a_pole={0: 1e-4, 1: 1e-3}, a_pole_elec={1: 2e6}, b_pole_elec={0: -2e5}))
    E.append(L.Element("sbend", "BFULLG0", {"l": 0.5, "k1": 0.08, "e1": 0.05, "e2": -0.04, "fint": 0.4,
                                            "hgap": 0.02}, fringe_type="full"))
    # fringe_type none with electric multipoles: the electric longitudinal
    # fringe alone at the ends
    E.append(L.Element("sbend", "BELECNONE", {"l": 0.7, "g": 0.012, "e1": 0.04}, fringe_type="none",
                       b_pole_elec={0: 1e4, 2: 3e7}))
    # collimator momentum and longitudinal limits: the ecollimator's (px, py)
    # ellipse and a single z limit, an rcollimator with no transverse limits
    E.append(L.Element("ecollimator", "ECMOM", {"l": 0.1, "x1_limit": 0.03, "x2_limit": 0.03, "y1_limit": 0.02,
                                                "y2_limit": 0.02, "px_aperture_width2": 1.2e-3,
                                                "py_aperture_width2": 6e-4, "px_aperture_center": 1e-4,
                                                "z_aperture_width2": 0.013}))
    E.append(L.Element("rcollimator", "RCMOM", {"l": 0.1, "pz_aperture_width2": 0.011, "pz_aperture_center": 5e-4,
                                                "py_aperture_width2": 7e-4}))
    # apertures that move with a bend (offset_moves_aperture): the curved
    # misaligned geometry, a bare ref_tilt and the straight (g = 0) geometry
    ap = {"x1_limit": 0.012, "x2_limit": 0.013, "y1_limit": 0.006, "y2_limit": 0.0065}
    E.append(L.Element("sbend", "BMISAP", {"l": 0.9, "g": 0.015, "e1": 0.02, "x_offset": 4e-4, "y_offset": -3e-4,
                                           "z_offset": 2e-3, "x_pitch": 2e-4, "y_pitch": 1e-4, "ref_tilt": 0.07,
                                           **ap}, offset_moves_aperture=True, aperture_at="both_ends"))
    E.append(L.Element("sbend", "BTILTAP", {"l": 0.6, "g": 0.01, "ref_tilt": 0.3, **ap}, offset_moves_aperture=True,
                       aperture_type="elliptical", aperture_at="both_ends"))
    E.append(L.Element("sbend", "BSTRAP", {"l": 0.5, "k1": 0.05, "x_offset": 5e-4, "y_pitch": 2e-4, **ap},
                       offset_moves_aperture=True, aperture_at="both_ends"))
    lat = L.Lattice(E, L.Species("electron", L.M_ELECTRON, -1), rings.p0c(), rings.E_TOT, "rare_zoo")
    return lat.finalize()


def random_particles(n: int, seed: int, scale: float = 1.0) -> np.ndarray:
    """Particles spanning a few mm / mrad / percent: (6, n)."""
    rng = np.random.Generator(np.random.Philox(seed))
    s = np.array([3e-3, 3e-4, 2e-3, 2e-4, 5e-3, 5e-3]) * scale
    return rng.standard_normal((6, n)) * s[:, None]


def rel_err(g: np.ndarray, o: np.ndarray, mask=None) -> np.ndarray:
    """Per-coordinate max of |g - o| / (|o| + rms_c)."""
    if mask is not None:
        g, o = g[:, mask], o[:, mask]
    if g.shape[1] == 0:
        return np.zeros(6)
    rms = np.sqrt(np.mean(o * o, axis=1))
    return np.max(np.abs(g - o) / (np.abs(o) + rms[:, None] + 1e-300), axis=1)


def oracle_track_elements(lat: L.Lattice, vec6: np.ndarray, start: int, stop: int, n_turns: int = 1,
                          threads: int = 0, variant: str = "glibc"):
    """Oracle over elements [start, stop) (turn loop when n_turns > 1).
    variant "glibc" evaluates transcendentals with the C library, as the
    reference does; "cr" rounds them correctly (the device's contract)."""
    from oracle import oracle as O

    lib = O.load(variant=variant)
    sub = L.Lattice(lat.elements[start:stop], lat.species, lat.p0c, lat.e_tot)
    eles = (O.Ele * len(sub.elements))()
    for i, e in enumerate(sub.elements):
        eles[i] = O.to_ele(e, lib)
    param = O.make_param(lat.species.mass, lat.species.charge)
    v = np.ascontiguousarray(vec6, dtype=np.float64).copy()
    n = v.shape[1]
    b = O.beta_of(lat.p0c, v[5], lat.species.mass)
    st = np.ones(n, np.int32)
    ie = np.full(n, -1, np.int32)
    it = np.full(n, -1, np.int32)
    O.track_turns(eles, lat.p0c, param, v, b, st, ie, it, n_turns, n_threads=threads, lib=lib)
    return v, b, st, ie, it


def oracle_batch_one_turn(lattices, variant: str = "cr"):
    """(vec6[6, m], variant[m]) -> vec6 after one turn, through the oracle,
    each particle in its own variant's lattice."""
    from oracle import oracle as O

    lib = O.load(variant=variant)
    eles = [O.to_eles(lat, lib) for lat in lattices]
    lat0 = lattices[0]
    param = O.make_param(lat0.species.mass, lat0.species.charge)

    def f(vec6, var):
        out = np.array(vec6, dtype=np.float64, copy=True)
        for v in np.unique(var):
            idx = np.nonzero(var == v)[0]
            sub = np.ascontiguousarray(out[:, idx])
            n = sub.shape[1]
            beta = O.beta_of(lat0.p0c, sub[5], lat0.species.mass)
            st = np.ones(n, np.int32)
            ie = np.full(n, -1, np.int32)
            it = np.full(n, -1, np.int32)
            O.track_turns(eles[v], lat0.p0c, param, sub, beta, st, ie, it, 1, lib=lib)
            out[:, idx] = sub
        return out

    return f


def oracle_da_survival(lattices, ref, n_angle, angle_min, angle_max, n_radius, r_max, yscale, n_turns,
                       variant: str = "cr", threads: int = 0):
    """survive_turns[v, d, a, r] of a polar-grid scan through the oracle."""
    from bgt import da
    from oracle import oracle as O

    lib = O.load(variant=variant)
    lat0 = lattices[0]
    param = O.make_param(lat0.species.mass, lat0.species.charge)
    nv, nd = ref.shape[:2]
    out = np.zeros((nv, nd, n_angle, n_radius), np.int32)
    for v in range(nv):
        v6 = da.grid_initial_conditions(ref[v:v + 1], n_angle, angle_min, angle_max, n_radius, r_max, yscale)
        v6 = np.ascontiguousarray(v6)
        n = v6.shape[1]
        beta = O.beta_of(lat0.p0c, v6[5], lat0.species.mass)
        st = np.ones(n, np.int32)
        ie = np.full(n, -1, np.int32)
        it = np.full(n, -1, np.int32)
        O.track_turns(O.to_eles(lattices[v], lib), lat0.p0c, param, v6, beta, st, ie, it, n_turns,
                      n_threads=threads, lib=lib)
        surv = np.where(st == 1, n_turns, it)
        out[v] = surv.reshape(nd, n_angle, n_radius)
    return out


def result_digest(vec6, beta, state, ix_ele_lost, ix_turn_lost) -> str:
    """SHA-256 of a tracking result's bytes (coordinates, beta, state, loss
    element, loss turn): equal digests mean bit-identical results."""
    import hashlib

    h = hashlib.sha256()
    for a, dt in ((vec6, np.float64), (beta, np.float64), (state, np.int32), (ix_ele_lost, np.int32),
                  (ix_turn_lost, np.int32)):
        h.update(np.ascontiguousarray(a, dtype=dt).tobytes())
    return h.hexdigest()


def plain_rel_err(g: np.ndarray, o: np.ndarray) -> np.ndarray:
    """Per particle, the largest plain per-coordinate relative error
    max_c |g_c - o_c| / |o_c| (0 where the values are equal, inf where o_c is
    0 and g_c is not): "relative per coordinate" as the parity bounds state it, with no
    floor, so a coordinate passing near zero counts at its own size."""
    d = np.abs(np.asarray(g, np.float64) - np.asarray(o, np.float64))
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.where(d == 0, 0.0, d / np.abs(o))
    return np.max(r, axis=0)


def exceed_digest(idx: np.ndarray) -> str:
    """SHA-256 of a sorted index list (the particles above a bound)."""
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(np.sort(idx), dtype=np.int64).tobytes()).hexdigest()


# Full-size parity cases: the configuration's ring and beam at its own size.
# (name, lattice factory kwargs, beam spec name, particles, turns)
CONFIG_PARITY_CASES = {
    "config0": dict(apertures=False, beam="CONFIG0_BEAM", n=10_000, turns=1000),
    "config1": dict(apertures=True, beam="CONFIG1_BEAM", n=20_000, turns=1000),
}


def config_parity_inputs(name: str):
    """(lattice, vec6) of a full-size parity case."""
    c = CONFIG_PARITY_CASES[name]
    lat = rings.fodo_ring(apertures=c["apertures"])
    v0 = rings.gaussian_beam(getattr(rings, c["beam"]), n=c["n"])
    return lat, v0


def qp_fraction(lo: int, hi: int):
    """The exact value of binary128 bits (normal values and zero)."""
    from fractions import Fraction

    lo, hi = int(lo), int(hi)
    e = (hi >> 48) & 0x7FFF
    frac = ((hi & ((1 << 48) - 1)) << 64) | lo
    val = Fraction(0) if (e == 0 and frac == 0) else (1 + Fraction(frac, 1 << 112)) * Fraction(2) ** (e - 16383)
    return -val if hi >> 63 else val


def time_residual(z0, z1, beta0, beta1, t0_bits, t1_bits, ref_time_start, delta_ref_time):
    """The tracking_method_test's seventh column for a forward particle
    (tracking_method_test.f90:219-221): the change of z less c_light times the
    change of beta * (reference time - t) through the element, evaluated from
    the particle times' exact binary128 values (the reference evaluates it in
    real(qp)) and rounded to double."""
    from fractions import Fraction

    ref_time = ref_time_start + delta_ref_time  # ele%ref_time, real(rp)
    ref_time_in = ref_time - delta_ref_time
    inner = (Fraction(beta1) * (Fraction(ref_time) - qp_fraction(*t1_bits))
             - Fraction(beta0) * (Fraction(ref_time_in) - qp_fraction(*t0_bits)))
    return float(Fraction(z1 - z0) - Fraction(L.C_LIGHT) * inner)


def oracle_track_timed(lat: L.Lattice, vec6: np.ndarray, start: int, stop: int, n_turns: int = 1,
                       variant: str = "cr", absolute_time: bool = False, threads: int = 0):
    """oracle_track_elements carrying the particle time (quad precision in the
    oracle) from init_coord's start, t = 0 - z / (beta c_light); returns
    (vec6, beta, state, ix_ele_lost, ix_turn_lost, t bits (n, 2) uint64)."""
    from bgt import qp
    from oracle import oracle as O

    lib = O.load(variant=variant)
    sub = L.Lattice(lat.elements[start:stop], lat.species, lat.p0c, lat.e_tot)
    eles = (O.Ele * len(sub.elements))()
    for i, e in enumerate(sub.elements):
        eles[i] = O.to_ele(e, lib)
    param = O.make_param(lat.species.mass, lat.species.charge, absolute_time=absolute_time)
    v = np.ascontiguousarray(vec6, dtype=np.float64).copy()
    n = v.shape[1]
    b = O.beta_of(lat.p0c, v[5], lat.species.mass)
    t = qp.initial_time(v, b)
    st = np.ones(n, np.int32)
    ie = np.full(n, -1, np.int32)
    it = np.full(n, -1, np.int32)
    O.track_turns(eles, lat.p0c, param, v, b, st, ie, it, n_turns, n_threads=threads, lib=lib, t=t)
    return v, b, st, ie, it, t
