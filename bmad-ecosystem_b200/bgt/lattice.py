"""Lattice model for the bgt tracker: Bmad elements, bookkeeping, and the
synthetic rings the benchmarks run on.

An :class:`Element` carries the ``ele%value(...)`` attributes the
``bmad_standard`` path reads, under Bmad's attribute names, plus the user
multipoles (``a_pole``/``b_pole`` etc.).  :func:`bookkeeper` restates the
parts of Bmad's attribute bookkeeping the tracker depends on, and
:func:`multipole_ele_to_ab` / :func:`multipole_ele_to_kt` restate the
multipole conversions whose results the C ABI takes precomputed (the role a
Fortran caller fills by calling Bmad's own routines).

Reference routines restated here (paths relative to the Bmad project root):

* ``bmad/code/attribute_bookkeeper.f90:150-180`` (``has_misalign``) and
  ``:295-404`` (``ds_step`` / ``num_steps``), with PTC's ``check_bend``
  (``forest/code/So_fitting.f90:3504-3536``).
* ``bmad/code/multipole_ele_to_ab.f90:31-678`` and
  ``bmad/code/multipole_ele_to_kt.f90:29-95``,
  ``bmad/low_level/multipole1_ab_to_kt.f90``,
  ``bmad/low_level/multipole1_kt_to_ab.f90``.
* element defaults from ``bmad/parsing/set_ele_defaults.f90:35-36,298,317``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

# sim_utils/interfaces/physical_constants.f90:12-37
PI = 3.141592653589793238462643383279
TWOPI = 2 * PI
C_LIGHT = 2.99792458e8
M_ELECTRON = 0.51099895069e6
M_PROTON = 0.93827208943e9

N_POLE = 22  # n_pole_maxx + 1

# Bmad element keys (bmad/modules/bmad_struct.f90:1681-1695)
KEYS = {
    "drift": 1, "sbend": 2, "quadrupole": 3, "sextupole": 5, "rfcavity": 9, "marker": 14, "kicker": 15,
    "octupole": 17, "multipole": 19, "ab_multipole": 22, "monitor": 31, "instrument": 32, "hkicker": 33,
    "vkicker": 34, "rcollimator": 35, "ecollimator": 36, "pipe": 44, "thick_multipole": 67,
}
# fringe_type (bmad_struct.f90:164-168)
FRINGE = {"none": 1, "soft_edge_only": 2, "hard_edge_only": 3, "full": 4, "sad_full": 5, "linear_edge": 6,
          "basic_bend": 7}
# fringe_at / aperture_at (bmad_struct.f90:372)
ENDS = {"entrance_end": 1, "exit_end": 2, "both_ends": 3, "no_end": 4}
# aperture_type (bmad_struct.f90:157), 0 = none set
APERTURE = {"none": 0, "rectangular": 2, "elliptical": 3}

# coord_struct%state (bmad_struct.f90:522-527)
ALIVE, LOST, LOST_NEG_X, LOST_POS_X, LOST_NEG_Y, LOST_POS_Y, LOST_Z, LOST_PZ = 1, 2, 3, 4, 5, 6, 7, 8

_HKICK_KEYS = {"quadrupole", "sbend", "sextupole", "octupole", "thick_multipole", "rfcavity", "ecollimator",
               "rcollimator", "instrument", "monitor", "pipe", "kicker"}

_VALUE_NAMES = [
    "l", "k1", "k2", "k3", "g", "dg", "e1", "e2", "fint", "hgap", "fintx", "hgapx", "voltage", "phi0",
    "phi0_multipass", "rf_frequency", "coupler_strength", "p0c", "e_tot", "ds_step", "x_offset", "y_offset",
    "z_offset", "x_pitch", "y_pitch", "tilt", "ref_tilt", "roll", "hkick", "vkick", "kick", "x1_limit",
    "x2_limit", "y1_limit", "y2_limit", "r0_mag", "r0_elec", "coupler_angle", "coupler_phase", "fq1", "fq2",
    "px_aperture_width2", "px_aperture_center", "py_aperture_width2", "py_aperture_center", "z_aperture_width2",
    "z_aperture_center", "pz_aperture_width2", "pz_aperture_center",
]


def rbend_to_sbend(values: Dict[str, float]) -> Dict[str, float]:
    """An rbend given by its chord length ``l`` and ``g`` or ``angle`` as the
    sbend the parser makes of it (bmad/parsing/bmad_parser_mod.f90:5080-5198,
    fiducial_pt = none): the arc length, the bend angle, the edge angles each
    increased by half the bend angle, and g = angle / l."""
    v = dict(values)
    l_chord = float(v.pop("l", 0.0))
    angle = float(v.pop("angle", 0.0))
    g = float(v.get("g", 0.0))
    if g != 0 and angle != 0:
        raise ValueError("rbend: give g or angle, not both")
    length = 0.0
    if l_chord != 0:
        if angle != 0:
            length = l_chord * angle / (2.0 * math.sin(0.5 * angle))
        elif g != 0:
            a = 0.5 * l_chord * g
            if abs(a) >= 1:
                raise ValueError("rbend: g * l is too large to be physical")
            a = 2.0 * math.asin(a)
            length = l_chord * a / (2.0 * math.sin(0.5 * a))
        else:
            length = l_chord
    if length != 0 and angle != 0:
        g = angle / length
    elif g != 0:
        angle = g * length
    v["e1"] = float(v.get("e1", 0.0)) + 0.5 * angle
    v["e2"] = float(v.get("e2", 0.0)) + 0.5 * angle
    if angle != 0:
        g = angle / length
    v["g"] = g
    v["l"] = length
    return v


@dataclass
class Element:
    """One Bmad lattice element (a subset of ``ele_struct``)."""

    key: str
    name: str = ""
    values: Dict[str, float] = field(default_factory=dict)
    num_steps: int = 0
    is_on: bool = True
    fringe_type: Optional[str] = None
    fringe_at: str = "both_ends"
    aperture_type: Optional[str] = None
    aperture_at: str = "exit_end"
    offset_moves_aperture: Optional[bool] = None
    exact_multipoles: int = 0
    scale_multipoles: bool = True
    # user multipoles, by order: a_pole[n] (an), b_pole[n] (bn); for a
    # multipole element a_pole = knl, b_pole = tn, ksl_pole = ksl
    a_pole: Dict[int, float] = field(default_factory=dict)
    b_pole: Dict[int, float] = field(default_factory=dict)
    ksl_pole: Dict[int, float] = field(default_factory=dict)
    a_pole_elec: Dict[int, float] = field(default_factory=dict)
    b_pole_elec: Dict[int, float] = field(default_factory=dict)
    # set by bookkeeper(): derived flags, and the user-given num_steps /
    # ds_step before the defaults were applied
    has_misalign: bool = False
    ix_ele: int = 0
    user_num_steps: Optional[int] = None
    user_ds_step: Optional[float] = None
    # rfcavity: the ends with a coupler kick (set_ele_defaults.f90:309)
    coupler_at: str = "exit_end"

    def __post_init__(self):
        if self.key == "rbend":
            self.values = rbend_to_sbend(self.values)
            self.key = "sbend"
        if self.key not in KEYS:
            raise ValueError(f"unsupported element key {self.key!r}")
        if self.fringe_type is None:
            # set_ele_defaults.f90:36,298,315
            self.fringe_type = {"sbend": "basic_bend", "rfcavity": "full"}.get(self.key, "none")
        if self.aperture_type is None:
            self.aperture_type = "elliptical" if self.key == "ecollimator" else "rectangular"
        if self.offset_moves_aperture is None:
            self.offset_moves_aperture = self.key in ("rcollimator", "ecollimator")
        if self.key == "rfcavity" and self.num_steps == 0 and "ds_step" not in self.values:
            self.num_steps = 10  # set_ele_defaults.f90:317

    def v(self, name: str) -> float:
        return float(self.values.get(name, 0.0))

    def copy(self) -> "Element":
        e = Element(self.key, self.name, dict(self.values), self.num_steps, self.is_on, self.fringe_type,
                    self.fringe_at, self.aperture_type, self.aperture_at, self.offset_moves_aperture,
                    self.exact_multipoles, self.scale_multipoles, dict(self.a_pole), dict(self.b_pole),
                    dict(self.ksl_pole), dict(self.a_pole_elec), dict(self.b_pole_elec), self.has_misalign,
                    self.ix_ele, self.user_num_steps, self.user_ds_step, self.coupler_at)
        return e

    @property
    def has_mag_poles(self) -> bool:
        return bool(self.a_pole or self.b_pole or self.ksl_pole)

    @property
    def has_elec_poles(self) -> bool:
        return bool(self.a_pole_elec or self.b_pole_elec)


def _arr(d: Dict[int, float]) -> np.ndarray:
    a = np.zeros(N_POLE)
    for n, x in d.items():
        a[int(n)] = float(x)
    return a


def _max_nonzero(a, b=None, n=N_POLE) -> int:
    """sim_utils/math/max_nonzero.f90:19-45"""
    for i in range(n - 1, -1, -1):
        if a[i] != 0:
            return i
        if b is not None and b[i] != 0:
            return i
    return -1


def _factorial(n: int) -> float:
    f = 1.0
    for i in range(2, n + 1):
        f = f * i
    return f


def _powi(x: float, m: int) -> float:
    """x**m with the multiply order gfortran uses (repeated squaring)."""
    n = abs(m)
    y = x if n % 2 else 1.0
    n >>= 1
    while n:
        x = x * x
        if n % 2:
            y = y * x
        n >>= 1
    return 1.0 / y if m < 0 else y


def _sign_of(x: float) -> int:
    return -1 if x < 0 else 1


def multipole1_ab_to_kt(an: float, bn: float, n: int):
    """bmad/low_level/multipole1_ab_to_kt.f90"""
    if an == 0 and bn == 0:
        return 0.0, 0.0
    knl = _factorial(n) * math.sqrt(an * an + bn * bn)
    tn = -math.atan2(an, bn) / (n + 1)
    if 2 * (n + 1) * abs(tn) > PI:
        knl = -knl
        tn = _sign_of(tn) * (abs(tn) - PI / (n + 1))
    return knl, tn


def multipole1_kt_to_ab(knl: float, knsl: float, tn: float, n: int):
    """bmad/low_level/multipole1_kt_to_ab.f90"""
    if knl == 0 and knsl == 0:
        return 0.0, 0.0
    angle = -tn * (n + 1)
    bn = (knl * math.cos(angle) - knsl * math.sin(angle)) / _factorial(n)
    an = (knl * math.sin(angle) + knsl * math.cos(angle)) / _factorial(n)
    return an, bn


def _tilt_this_multipole(ele: Element, sgn: int, a, b, ix: int):
    """multipole_ele_to_ab.f90:436-457"""
    tilt = sgn * (ele.v("ref_tilt") if ele.key == "sbend" else ele.v("tilt"))
    if tilt == 0:
        return
    for n in range(ix + 1):
        if a[n] == 0 and b[n] == 0:
            continue
        an, bn = a[n], b[n]
        c = math.cos((n + 1) * tilt)
        s = math.sin((n + 1) * tilt)
        b[n] = bn * c + an * s
        a[n] = -bn * s + an * c


def _convert_this_ab(ele: Element, electric: bool):
    """multipole_ele_to_ab.f90:463-575 (non-slave: zero relative tilt,
    field_master = F)."""
    a = _arr(ele.a_pole_elec if electric else ele.a_pole)
    b = _arr(ele.b_pole_elec if electric else ele.b_pole)
    if _max_nonzero(a, b) < 0 or not ele.scale_multipoles:
        return a, b
    if electric:
        radius = ele.v("r0_elec")
        if radius != 0 and radius != 1:
            factor = radius
            for n in range(N_POLE):
                factor = factor / radius
                a[n] = factor * a[n]
                b[n] = factor * b[n]
        return a, b
    key = ele.key
    if key == "sbend":
        const, ref_exp = ele.v("l") * (ele.v("g") + ele.v("dg")), 0
    elif key == "kicker":
        hk, vk = ele.v("hkick"), ele.v("vkick")
        const = vk if hk == 0 else (hk if vk == 0 else math.sqrt(hk * hk + vk * vk))
        ref_exp = 0
    elif key in ("hkicker", "vkicker"):
        const, ref_exp = ele.v("kick"), 0
    elif key == "quadrupole":
        const, ref_exp = ele.v("k1") * ele.v("l"), 1
    elif key == "sextupole":
        const, ref_exp = ele.v("k2") * ele.v("l"), 2
    elif key == "octupole":
        const, ref_exp = ele.v("k3") * ele.v("l"), 3
    elif key in ("ab_multipole", "thick_multipole", "rfcavity"):
        return a, b
    else:
        raise ValueError(f"{ele.name}: trying to scale multipoles of a non-scalable element ({key})")
    radius = ele.v("r0_mag")
    if radius == 0:
        a = const * a
        b = const * b
    else:
        factor = const * _powi(radius, ref_exp + 1)
        for n in range(N_POLE):
            factor = factor / radius
            a[n] = factor * a[n]
            b[n] = factor * b[n]
    return a, b


def _non_multipoles(ele: Element, electric: bool):
    """this_ele_non_multipoles, multipole_ele_to_ab.f90:324-410"""
    ak = np.zeros(4)
    bk = np.zeros(4)
    if electric:
        return ak, bk
    key = ele.key
    if key == "hkicker":
        bk[0] = -ele.v("kick")
    elif key == "vkicker":
        ak[0] = ele.v("kick")
    elif key == "kicker":
        bk[0] = -ele.v("hkick")
        ak[0] = ele.v("vkick")
    else:
        hk, vk = ele.v("hkick"), ele.v("vkick")
        if key in _HKICK_KEYS and (hk != 0 or vk != 0):
            tilt = ele.v("ref_tilt") if key == "sbend" else ele.v("tilt")
            if tilt != 0:
                c, s = math.cos(tilt), math.sin(tilt)
                bk[0] = -hk * c - vk * s
                ak[0] = -hk * s + vk * c
            else:
                bk[0] = -hk
                ak[0] = vk
    if key == "quadrupole":
        bk[1] = ele.v("k1") * ele.v("l")
    elif key == "sbend":
        bk[0] = bk[0] + ele.v("dg") * ele.v("l")
        bk[1] = ele.v("k1") * ele.v("l")
        bk[2] = ele.v("k2") * ele.v("l") / 2.0
    elif key == "sextupole":
        bk[2] = ele.v("k2") * ele.v("l") / 2.0
    elif key == "octupole":
        bk[3] = ele.v("k3") * ele.v("l") / 6.0
    return ak, bk


def multipole_ele_to_ab(ele: Element, use_ele_tilt: bool = False, electric: bool = False,
                        include_kicks: bool = True):
    """Restates ``multipole_ele_to_ab`` (non-slave path) without pulling b1.
    Returns (ix_pole_max, a, b)."""
    a = np.zeros(N_POLE)
    b = np.zeros(N_POLE)
    if not ele.is_on or ele.key == "pipe":
        return -1, a, b
    if ele.key == "multipole":
        if electric or not ele.has_mag_poles:
            return -1, a, b
        knl, tn, ksl = _arr(ele.a_pole), _arr(ele.b_pole), _arr(ele.ksl_pole)
        for n in range(N_POLE):
            a[n], b[n] = multipole1_kt_to_ab(knl[n], ksl[n], tn[n], n)
        return _max_nonzero(a, b), a, b
    has = ele.has_elec_poles if electric else ele.has_mag_poles
    if has:
        a, b = _convert_this_ab(ele, electric)
    ak, bk = _non_multipoles(ele, electric)
    if include_kicks:
        for i in range(4):
            a[i] = a[i] + ak[i]
            b[i] = b[i] + bk[i]
    ix = _max_nonzero(a, b)
    if use_ele_tilt:
        _tilt_this_multipole(ele, +1, a, b, ix)
    return ix, a, b


def multipole_ele_to_kt(ele: Element, use_ele_tilt: bool = True):
    """Restates ``multipole_ele_to_kt`` (magnetic).  Returns (ix, knl, tn)."""
    knl = np.zeros(N_POLE)
    tn = np.zeros(N_POLE)
    if ele.key == "multipole":
        if not ele.has_mag_poles:
            return -1, knl, tn
        kp, tp, ks = _arr(ele.a_pole), _arr(ele.b_pole), _arr(ele.ksl_pole)
        if not np.any(ks != 0):
            knl = kp.copy()
            tn = tp + ele.v("tilt")
        else:
            for n in range(N_POLE):
                knl[n] = math.sqrt(kp[n] ** 2 + ks[n] ** 2)
                tn[n] = tp[n] - math.atan2(ks[n], kp[n]) / (n + 1)
                if 2 * (n + 1) * abs(tn[n]) > PI:
                    knl[n] = -knl[n]
                    tn[n] = _sign_of(tn[n]) * (abs(tn[n]) - PI / (n + 1))
        return _max_nonzero(knl), knl, tn
    ix, a, b = multipole_ele_to_ab(ele, use_ele_tilt, False, include_kicks=False)
    if ix > -1:
        for n in range(N_POLE):
            knl[n], tn[n] = multipole1_ab_to_kt(a[n], b[n], n)
    return ix, knl, tn


def check_bend(xl: float, ggi: float, rhoi: float, xbend1: float):
    """PTC check_bend, forest/code/So_fitting.f90:3504-3536.  Returns (met, gf)."""
    gg = float(int(ggi))
    if gg == 0:
        gg = 1.0
    co = [0.0] * 8
    co[2], co[4], co[6] = 1.0 / 12.0, 0.17, 0.17e-1
    gf = [0.0] * 8
    for i in (3, 5, 7):
        ar = i - 1
        gf[i] = (co[i - 1] / xbend1) ** (1.0 / ar) * abs(rhoi) * xl
        if gf[i] < gg:
            gf[i] = gg
    gf[2] = gf[3]
    gf[4] = gf[5] * 3
    gf[6] = gf[7] * 7
    met = 2
    if gf[4] < gf[2]:
        met = 4
    if gf[6] < gf[4] and gf[6] < gf[2]:
        met = 6
    return met, gf


def _nint(x: float) -> int:
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


def bookkeeper(ele: Element) -> Element:
    """attribute_bookkeeper.f90:150-180 and :295-404 (see module docstring)."""
    v = ele.values
    if ele.user_num_steps is None:
        ele.user_num_steps = ele.num_steps
        ele.user_ds_step = float(v.get("ds_step", 0.0))
    if ele.key == "sbend":
        mis = ele.v("ref_tilt") != 0 or ele.v("roll") != 0
    else:
        mis = ele.v("tilt") != 0
    ele.has_misalign = bool(mis or any(ele.v(n) != 0 for n in
                                        ("x_offset", "y_offset", "z_offset", "x_pitch", "y_pitch")))
    if "fintx" not in v:
        v["fintx"] = ele.v("fint")
    if "hgapx" not in v:
        v["hgapx"] = ele.v("hgap")
    if ele.key in ("marker", "multipole", "ab_multipole") or ele.v("p0c") <= 0:
        return ele
    L = ele.v("l")
    if ele.v("ds_step") == 0 and ele.num_steps == 0:
        if ele.key in ("drift", "pipe", "ecollimator", "rcollimator", "instrument", "monitor"):
            ele.num_steps = 1
            v["ds_step"] = L
        elif ele.key in ("sbend", "quadrupole", "sextupole") and L != 0:
            ix, knl, _ = multipole_ele_to_kt_for_steps(ele)
            knl = np.abs(knl)
            bend_factor = knl[0] / L
            radius0 = ele.v("r0_mag") or 0.01
            if ele.key == "sbend":
                bend_factor = bend_factor + max(abs(ele.v("g")), abs(ele.v("g") + ele.v("dg")))
                quad_factor = knl[1] + knl[2] * radius0 + L * bend_factor ** 2
            elif ele.key == "quadrupole":
                quad_factor = 50 * (knl[1] + L * bend_factor ** 2)
            else:
                quad_factor = knl[2] * radius0 + L * bend_factor ** 2
            if ele.has_elec_poles:
                r0e = ele.v("r0_elec") or 0.01
                _, ae, be = multipole_ele_to_ab(ele, False, True, False)
                bend_factor = bend_factor + (abs(ae[0]) + abs(be[0])) / ele.v("p0c")
                quad_factor = quad_factor + (abs(ae[1]) + abs(be[1]) + r0e * (abs(ae[2]) + abs(be[2]))) / ele.v("p0c")
            met, gf = check_bend(L, quad_factor, bend_factor, 1e-8)
            met = min(met, 4)
            ele.num_steps = max(_nint(gf[met + 1]), 1)
            v["ds_step"] = abs(L) / ele.num_steps
        elif ele.key in ("kicker", "hkicker", "vkicker") and L != 0:
            if ele.key == "kicker":
                km = math.sqrt(ele.v("hkick") ** 2 + ele.v("vkick") ** 2) / L
            else:
                km = ele.v("kick") / L
            met, gf = check_bend(L, 0.0, km, 1e-8)
            ele.num_steps = max(_nint(gf[met + 1]), 1)
            v["ds_step"] = abs(L) / ele.num_steps
    if ele.v("ds_step") <= 0:
        if ele.num_steps <= 0 or abs(L) == 0:
            v["ds_step"] = 0.2  # bmad_com%default_ds_step
        else:
            v["ds_step"] = abs(L) / ele.num_steps
    ele.num_steps = max(1, _nint(abs(L / ele.v("ds_step"))))
    return ele


def multipole_ele_to_kt_for_steps(ele: Element):
    """multipole_ele_to_kt(ele, .false., ix, knl, tilt, magnetic$, include_kicks$)
    as called by the num_steps bookkeeping."""
    ix, a, b = multipole_ele_to_ab(ele, False, False, include_kicks=True)
    knl = np.zeros(N_POLE)
    tn = np.zeros(N_POLE)
    for n in range(N_POLE):
        knl[n], tn[n] = multipole1_ab_to_kt(a[n], b[n], n)
    return ix, knl, tn


@dataclass
class Species:
    name: str = "electron"
    mass: float = M_ELECTRON
    charge: int = -1


@dataclass
class Lattice:
    """A ring: elements 1..N (ix_ele), one species, one reference momentum."""

    elements: List[Element]
    species: Species = field(default_factory=Species)
    p0c: float = 0.0
    e_tot: float = 0.0
    name: str = ""
    info: Dict[str, float] = field(default_factory=dict)

    def finalize(self) -> "Lattice":
        ref_time = 0.0
        for i, e in enumerate(self.elements):
            e.ix_ele = i + 1
            e.values["p0c"] = self.p0c
            e.values["e_tot"] = self.e_tot
            bookkeeper(e)
            # reference time at the entrance and through the element, as
            # lat_compute_reference_energy.f90 computes them for an element
            # with a constant reference velocity (:743-748: delta_ref_time =
            # l * E_tot / (p0c * c_light), 0 for zero length; ref_time =
            # ref_time_start + delta_ref_time).  For an rfcavity Bmad tracks
            # the reference particle instead (:750-753), which gives the same
            # time up to rounding when the cavity does not change the
            # reference energy; a caller with Bmad passes Bmad's own values.
            e.values["ref_time_start"] = ref_time
            ln = e.v("l")
            dt = 0.0 if (ln == 0 or e.key == "marker") else ln * self.e_tot / (self.p0c * C_LIGHT)
            e.values["delta_ref_time"] = dt
            ref_time = ref_time + dt
        return self

    @property
    def circumference(self) -> float:
        return sum(e.v("l") for e in self.elements)

    def __len__(self):
        return len(self.elements)


def p0c_from_e_tot(e_tot: float, mass: float) -> float:
    return math.sqrt(e_tot * e_tot - mass * mass)


def beta_of(p0c: float, pz, mass: float):
    """convert_pc_to (beta = pc / sqrt(pc**2 + mc2**2))"""
    pc = (1 + np.asarray(pz, dtype=np.float64)) * p0c
    return pc / np.sqrt(pc * pc + mass * mass)
