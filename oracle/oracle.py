"""Python binding of the CPU oracle (bmad_oracle.c).  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module, as the checker and the timed CPU baseline.  The product
(bmad-ecosystem_b200/) never imports it.

The oracle restates the reference's bmad_standard tracking in C; this module
converts the product's Element descriptions (raw Bmad attributes and user
multipoles) into the oracle's element struct.  The oracle then does its own
multipole bookkeeping (multipole_ele_to_ab) independently of the product.
"""
from __future__ import annotations

import ctypes as C
import math
import struct
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
N_POLE = 22

KEY = {"drift": 1, "quadrupole": 2, "sbend": 3, "sextupole": 4, "octupole": 5, "thick_multipole": 6,
       "multipole": 7, "ab_multipole": 8, "rfcavity": 9, "marker": 10, "ecollimator": 11, "rcollimator": 12,
       "instrument": 13, "monitor": 14, "pipe": 15, "hkicker": 16, "vkicker": 17, "kicker": 18}
FRINGE = {"none": 0, "basic_bend": 1, "full": 2, "hard_edge_only": 3, "soft_edge_only": 4, "sad_full": 5,
          "linear_edge": 6}
ENDS = {"no_end": 0, "entrance_end": 1, "exit_end": 2, "both_ends": 3}
APT = {"rectangular": 0, "elliptical": 1, "none": 0}


class Param(C.Structure):
    _fields_ = [("mass", C.c_double), ("charge", C.c_int), ("max_aperture_limit", C.c_double),
                ("aperture_limit_on", C.c_int), ("unstable_factor", C.c_double),
                ("absolute_time_tracking", C.c_int), ("absolute_time_ref_shift", C.c_int)]


class Coord(C.Structure):
    # t is the C struct's __float128 (16 bytes, 16-byte aligned); c_longdouble
    # has that size and alignment on x86-64 and only reserves the space here
    _fields_ = [("vec", C.c_double * 6), ("beta", C.c_double), ("p0c", C.c_double), ("state", C.c_int),
                ("t_qp", C.c_longdouble)]


_INTS = ["key", "ix_ele", "is_on", "fringe_type", "fringe_at", "aperture_type", "aperture_at",
         "offset_moves_aperture", "has_mag_poles", "has_elec_poles", "scale_multipoles", "field_master",
         "has_misalign", "num_steps", "coupler_at"]
_DBLS = ["l", "k1", "k2", "k3", "g", "dg", "e1", "e2", "fint", "hgap", "fintx", "hgapx", "voltage", "phi0",
         "phi0_multipass", "rf_frequency", "p0c", "e_tot", "ds_step", "x_offset", "y_offset", "z_offset", "x_pitch",
         "y_pitch", "tilt", "ref_tilt", "roll", "hkick", "vkick", "kick", "x1_limit", "x2_limit", "y1_limit",
         "y2_limit", "px_aperture_width2", "px_aperture_center", "py_aperture_width2", "py_aperture_center",
         "z_aperture_width2", "z_aperture_center", "pz_aperture_width2", "pz_aperture_center", "r0_mag", "r0_elec",
         "coupler_strength", "coupler_angle", "coupler_phase", "fq1", "fq2", "delta_ref_time", "ref_time_start"]


class Ele(C.Structure):
    _fields_ = [(n, C.c_int) for n in _INTS] + [(n, C.c_double) for n in _DBLS] + [
        (n, C.c_double * N_POLE) for n in ("a_pole", "b_pole", "ksl_pole", "a_pole_elec", "b_pole_elec")]


_libs = {}
VARIANTS = {"glibc": "liboracle.so", "count": "liboracle_count.so", "cr": "liboracle_cr.so"}


def build():
    """Compile the oracle libraries (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def _bind(lib):
    lib.bgo_ele_init.argtypes = [C.POINTER(Ele), C.c_int]
    lib.bgo_bookkeeper.argtypes = [C.POINTER(Ele)]
    lib.bgo_multipole_ele_to_ab.argtypes = [C.POINTER(Ele), C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double),
                                            C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.bgo_multipole_ele_to_kt.argtypes = [C.POINTER(Ele), C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.bgo_init_coord.argtypes = [C.POINTER(Coord), C.POINTER(C.c_double), C.c_double, C.POINTER(Param)]
    lib.bgo_track1.argtypes = [C.POINTER(Coord), C.POINTER(Ele), C.POINTER(Param)]
    lib.bgo_check_aperture_limit.argtypes = [C.POINTER(Coord), C.POINTER(Ele), C.c_int, C.POINTER(Param)]
    lib.bgo_hwang_bend_edge_kick.argtypes = [C.POINTER(Ele), C.c_int, C.POINTER(Coord), C.POINTER(Param)]
    lib.bgo_orbit_too_large.argtypes = [C.POINTER(Coord), C.POINTER(Param)]
    lib.bgo_offset_particle.argtypes = [C.POINTER(Ele), C.c_int, C.POINTER(Coord), C.c_int, C.c_double,
                                        C.POINTER(Param), C.POINTER(C.c_double)]
    lib.bgo_track_turns.argtypes = [C.POINTER(Ele), C.c_int, C.POINTER(Param), C.c_double, C.POINTER(C.c_double),
                                    C.POINTER(C.c_double), C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                    C.POINTER(C.c_int), C.c_long, C.c_int, C.c_int, C.c_int, C.c_int]
    lib.bgo_flop_counter_read.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.bgo_c_multi.argtypes = [C.c_int, C.c_int, C.c_int]
    lib.bgo_c_multi.restype = C.c_double
    return lib


def load(count_flops: bool = False, variant: str = "glibc"):
    """The oracle library.  variant "glibc": transcendentals from the C library,
    as the reference evaluates them; "cr": transcendentals of particle
    coordinates correctly rounded; "count": glibc build with FP64 operation
    counters (single thread)."""
    if count_flops:
        variant = "count"
    if variant not in _libs:
        path = BUILD / VARIANTS[variant]
        if not path.exists():
            build()
        _libs[variant] = _bind(C.CDLL(str(path)))
    return _libs[variant]


def make_param(mass: float, charge: int = -1, aperture_limit_on: bool = True, absolute_time: bool = False,
               absolute_time_ref_shift: bool = True) -> Param:
    return Param(mass, charge, 1e3, 1 if aperture_limit_on else 0, 0.0, 1 if absolute_time else 0,
                 1 if absolute_time_ref_shift else 0)


def to_ele(e, lib=None, raw_bookkeeping: bool = False) -> Ele:
    """Convert a product Element (bgt.lattice.Element) to the oracle struct.
    The bookkeeping results (num_steps, ds_step, has_misalign) are recomputed
    by the oracle's own bookkeeper."""
    lib = lib or load()
    o = Ele()
    lib.bgo_ele_init(C.byref(o), KEY[e.key])
    o.ix_ele = e.ix_ele
    o.is_on = 1 if e.is_on else 0
    o.fringe_type = FRINGE[e.fringe_type]
    o.fringe_at = ENDS[e.fringe_at]
    o.aperture_type = APT[e.aperture_type]
    o.aperture_at = ENDS[e.aperture_at]
    o.offset_moves_aperture = 1 if e.offset_moves_aperture else 0
    o.coupler_at = ENDS[getattr(e, "coupler_at", "exit_end")]
    o.scale_multipoles = 1 if e.scale_multipoles else 0
    for n in _DBLS:
        if n in e.values:
            setattr(o, n, float(e.values[n]))
    if "fintx" not in e.values:
        o.fintx = float("nan")
    if "hgapx" not in e.values:
        o.hgapx = float("nan")
    # the oracle redoes the num_steps / ds_step bookkeeping from the user inputs
    o.num_steps = int(e.user_num_steps if e.user_num_steps is not None else e.num_steps)
    o.ds_step = float(e.user_ds_step if e.user_ds_step is not None else e.values.get("ds_step", 0.0))
    for arr, d in (("a_pole", e.a_pole), ("b_pole", e.b_pole), ("ksl_pole", e.ksl_pole),
                   ("a_pole_elec", e.a_pole_elec), ("b_pole_elec", e.b_pole_elec)):
        a = getattr(o, arr)
        for n, x in d.items():
            a[int(n)] = float(x)
    o.has_mag_poles = 1 if (e.a_pole or e.b_pole or e.ksl_pole) else 0
    o.has_elec_poles = 1 if (e.a_pole_elec or e.b_pole_elec) else 0
    lib.bgo_bookkeeper(C.byref(o))
    return o


def to_eles(lattice, lib=None):
    lib = lib or load()
    arr = (Ele * len(lattice.elements))()
    for i, e in enumerate(lattice.elements):
        arr[i] = to_ele(e, lib)
    return arr


def track1(ele: Ele, vec6, p0c: float, param: Param, beta=None, state: int = 1, lib=None):
    """Single particle through one element; returns (vec6, beta, state)."""
    lib = lib or load()
    c = Coord()
    v = (C.c_double * 6)(*[float(x) for x in vec6])
    lib.bgo_init_coord(C.byref(c), v, p0c, C.byref(param))
    if beta is not None:
        c.beta = beta
    c.state = state
    lib.bgo_track1(C.byref(c), C.byref(ele), C.byref(param))
    return np.array(c.vec[:]), c.beta, c.state


def coord_time_bits(c: Coord):
    """The binary128 bits (lo, hi) of a Coord's time t."""
    lo, hi = struct.unpack("<QQ", C.string_at(C.addressof(c) + Coord.t_qp.offset, 16))
    return lo, hi


def track1_timed(ele: Ele, vec6, p0c: float, param: Param, lib=None):
    """track1 from init_coord's start (t = 0 - z / (beta c_light)); returns
    (vec6, beta, state, start beta, start t bits, end t bits)."""
    lib = lib or load()
    c = Coord()
    v = (C.c_double * 6)(*[float(x) for x in vec6])
    lib.bgo_init_coord(C.byref(c), v, p0c, C.byref(param))
    beta0, t0 = c.beta, coord_time_bits(c)
    lib.bgo_track1(C.byref(c), C.byref(ele), C.byref(param))
    return np.array(c.vec[:]), c.beta, c.state, beta0, t0, coord_time_bits(c)


def track_turns(eles, p0c: float, param: Param, vec6: np.ndarray, beta: np.ndarray, state: np.ndarray,
                ix_ele_lost: np.ndarray, ix_turn_lost: np.ndarray, n_turns: int, turn0: int = 0,
                n_threads: int = 0, element_outer: bool = False, lib=None, t: np.ndarray = None):
    """Multi-turn tracking in place.  vec6 is (6, n) C-contiguous float64; t
    (optional) the particle times as binary128 bits, a C-contiguous (n, 2)
    uint64 array (bgt.qp's layout), carried in quad precision like the
    reference's real(qp) coord_struct%t."""
    lib = lib or load()
    n = vec6.shape[1]
    assert vec6.flags["C_CONTIGUOUS"] and vec6.dtype == np.float64
    if t is not None:
        assert t.shape == (n, 2) and t.flags["C_CONTIGUOUS"] and t.dtype == np.uint64
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    lib.bgo_track_turns(eles, len(eles), C.byref(param), p0c, vec6.ctypes.data_as(dp), beta.ctypes.data_as(dp),
                        t.ctypes.data if t is not None else None, state.ctypes.data_as(ip),
                        ix_ele_lost.ctypes.data_as(ip), ix_turn_lost.ctypes.data_as(ip), n, turn0, n_turns,
                        n_threads, 1 if element_outer else 0)


def beta_of(p0c, pz, mass):
    pc = (1 + np.asarray(pz, dtype=np.float64)) * p0c
    return pc / np.sqrt(pc * pc + mass * mass)


def one_turn_fn(lattice, n_threads: int = 0, lib=None):
    """A one-turn map (6, n) -> (6, n) through the oracle, for optics."""
    lib = lib or load()
    eles = to_eles(lattice, lib)
    param = make_param(lattice.species.mass, lattice.species.charge)

    def f(v):
        v = np.ascontiguousarray(v, dtype=np.float64)
        n = v.shape[1]
        b = beta_of(lattice.p0c, v[5], lattice.species.mass)
        st = np.ones(n, np.int32)
        ie = np.full(n, -1, np.int32)
        it = np.full(n, -1, np.int32)
        track_turns(eles, lattice.p0c, param, v, b, st, ie, it, 1, n_threads=n_threads, lib=lib)
        return v

    return f


def flops_per_particle_turn(lattice, vec6: np.ndarray, n_turns: int = 1):
    """FP64 operations (and libm calls) per particle per turn, counted by the
    instrumented oracle build over the given particles."""
    lib = load(count_flops=True)
    eles = to_eles(lattice, lib)
    param = make_param(lattice.species.mass, lattice.species.charge)
    v = np.ascontiguousarray(vec6, dtype=np.float64).copy()
    n = v.shape[1]
    b = beta_of(lattice.p0c, v[5], lattice.species.mass)
    st = np.ones(n, np.int32)
    ie = np.full(n, -1, np.int32)
    it = np.full(n, -1, np.int32)
    lib.bgo_flop_counter_reset()
    track_turns(eles, lattice.p0c, param, v, b, st, ie, it, n_turns, n_threads=1, lib=lib)
    fl = C.c_double()
    lm = C.c_double()
    lib.bgo_flop_counter_read(C.byref(fl), C.byref(lm))
    return fl.value / (n * n_turns), lm.value / (n * n_turns)
