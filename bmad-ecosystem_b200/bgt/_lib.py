"""ctypes binding to libbgt.so (the C ABI in include/bgt.h).

The library is built in-tree (``bmad-ecosystem_b200/build.py``).  Loading
fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import lattice as L

N_POLE = L.N_POLE
_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libbgt.so"

# error codes (bgt.h)
BGT_OK, BGT_EINVAL, BGT_EUNSUPPORTED, BGT_ECUDA, BGT_ENOMEM, BGT_ETIMEOUT, BGT_ETOOLARGE = 0, -1, -2, -3, -4, -5, -6


class BgtElement(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "key", "ix_ele", "is_on", "num_steps", "fringe_type", "fringe_at", "aperture_type", "aperture_at",
        "offset_moves_aperture", "exact_multipoles", "has_misalign", "coupler_at")] + [
        (n, C.c_double) for n in (
            "l", "k1", "k2", "k3", "g", "dg", "e1", "e2", "fint", "hgap", "fintx", "hgapx", "voltage", "phi0",
            "phi0_multipass", "rf_frequency", "coupler_strength", "p0c", "e_tot", "ds_step", "x_offset",
            "y_offset", "z_offset", "x_pitch", "y_pitch", "tilt", "ref_tilt", "roll", "hkick", "vkick", "kick",
            "x1_limit", "x2_limit", "y1_limit", "y2_limit")] + [
        (n, C.c_double * N_POLE) for n in ("an", "bn", "an_elec", "bn_elec", "knl", "tn")] + [
        ("coupler_angle", C.c_double), ("coupler_phase", C.c_double), ("fq1", C.c_double), ("fq2", C.c_double)] + [
        (n, C.c_double) for n in ("px_aperture_width2", "px_aperture_center", "py_aperture_width2",
                                  "py_aperture_center", "z_aperture_width2", "z_aperture_center",
                                  "pz_aperture_width2", "pz_aperture_center", "delta_ref_time", "ref_time_start")]


class BgtSpecies(C.Structure):
    _fields_ = [("mass", C.c_double), ("charge", C.c_int32), ("aperture_limit_on", C.c_int32),
                ("max_aperture_limit", C.c_double), ("absolute_time_tracking", C.c_int32),
                ("absolute_time_ref_shift", C.c_int32)]


class BgtTuning(C.Structure):
    _fields_ = [("threads_per_block", C.c_int32), ("blocks_per_sm", C.c_int32), ("turns_per_launch", C.c_int32),
                ("compact_every", C.c_int32), ("table_mode", C.c_int32), ("wait_limit_us", C.c_int32),
                ("test_skip_table_copy", C.c_int32)]


class BgtError(RuntimeError):
    pass


_lib = None

# every symbol include/bgt.h and include/bgt_mlp.h declare
EXPORTED = [
    "bgt_create", "bgt_destroy", "bgt_last_error", "bgt_table_info", "bgt_set_tuning", "bgt_get_tuning",
    "bgt_track_turns", "bgt_track_turns_device", "bgt_device_status", "bgt_track_elements", "bgt_da_scan_grid",
    "bgt_kernel_launch_count", "bgt_fp64_peak_tflops", "bgt_track_turns_device_noalloc",
    # include/bgt_mlp.h
    "bgt_mlp_create", "bgt_mlp_destroy", "bgt_mlp_last_error", "bgt_mlp_launch_count", "bgt_mlp_get_params",
    "bgt_mlp_set_params", "bgt_mlp_forward", "bgt_mlp_gradients", "bgt_mlp_train_step", "bgt_mlp_features",
    "bgt_mlp_gemm_bf16", "bgt_mlp_gemm_bf16_wait_test",
]

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


def load() -> C.CDLL:
    """Load libbgt.so once.  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("BGT_LIBRARY", LIB_PATH))
    if not path.exists():
        raise BgtError(f"libbgt.so not found at {path}; build it with `python bmad-ecosystem_b200/build.py`")
    lib = C.CDLL(str(path))
    lib.bgt_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(BgtElement), C.c_int32, C.c_int32,
                               C.POINTER(BgtSpecies), C.c_int32]
    lib.bgt_create.restype = C.c_int
    lib.bgt_destroy.argtypes = [C.c_void_p]
    lib.bgt_last_error.argtypes = [C.c_void_p]
    lib.bgt_last_error.restype = C.c_char_p
    lib.bgt_table_info.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
    lib.bgt_set_tuning.argtypes = [C.c_void_p, C.POINTER(BgtTuning)]
    lib.bgt_get_tuning.argtypes = [C.c_void_p, C.POINTER(BgtTuning)]
    lib.bgt_track_turns.argtypes = [C.c_void_p, _dp, _dp, C.c_void_p, _ip, _ip, _ip, _ip, C.c_int64, C.c_int32,
                                    C.c_int32]
    lib.bgt_track_turns_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_void_p]
    lib.bgt_device_status.argtypes = [C.c_void_p, C.c_void_p]
    lib.bgt_track_elements.argtypes = [C.c_void_p, _dp, _dp, C.c_void_p, _ip, _ip, _ip, C.c_int64, C.c_int32,
                                       C.c_int32]
    lib.bgt_da_scan_grid.argtypes = [C.c_void_p, _dp, C.c_int32, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                     C.c_int32, C.c_double, C.c_double, C.c_int32, _dp, _ip]
    lib.bgt_kernel_launch_count.argtypes = [C.c_void_p]
    lib.bgt_kernel_launch_count.restype = C.c_int64
    lib.bgt_fp64_peak_tflops.argtypes = [C.c_int32, _dp]
    lib.bgt_track_turns_device_noalloc.argtypes = [
        C.POINTER(BgtElement), C.c_int32, C.POINTER(BgtSpecies), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
        C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.POINTER(BgtTuning), C.c_int32, C.c_void_p, C.c_void_p,
        C.c_char_p, C.c_int32]
    _lib = lib
    return lib


def to_bgt_element(e: L.Element) -> BgtElement:
    """Flatten an Element into the C struct, filling an/bn (and the electric
    pair) with multipole_ele_to_ab and knl/tn with multipole_ele_to_kt, as a
    Fortran caller would with Bmad's own routines."""
    b = BgtElement()
    b.key = L.KEYS[e.key]
    b.ix_ele = e.ix_ele
    b.is_on = 1 if e.is_on else 0
    b.num_steps = e.num_steps
    b.fringe_type = L.FRINGE[e.fringe_type]
    b.fringe_at = L.ENDS[e.fringe_at]
    b.aperture_type = L.APERTURE[e.aperture_type] if (e.aperture_type != "none") else 0
    b.aperture_at = L.ENDS[e.aperture_at]
    b.offset_moves_aperture = 1 if e.offset_moves_aperture else 0
    b.exact_multipoles = e.exact_multipoles
    b.has_misalign = 1 if e.has_misalign else 0
    b.coupler_at = L.ENDS[e.coupler_at]
    b.coupler_angle = e.v("coupler_angle")
    b.coupler_phase = e.v("coupler_phase")
    b.fq1 = e.v("fq1")
    b.fq2 = e.v("fq2")
    for n in ("l", "k1", "k2", "k3", "g", "dg", "e1", "e2", "fint", "hgap", "fintx", "hgapx", "voltage", "phi0",
              "phi0_multipass", "rf_frequency", "coupler_strength", "p0c", "e_tot", "ds_step", "x_offset",
              "y_offset", "z_offset", "x_pitch", "y_pitch", "tilt", "ref_tilt", "roll", "hkick", "vkick", "kick",
              "x1_limit", "x2_limit", "y1_limit", "y2_limit", "px_aperture_width2", "px_aperture_center",
              "py_aperture_width2", "py_aperture_center", "z_aperture_width2", "z_aperture_center",
              "pz_aperture_width2", "pz_aperture_center", "delta_ref_time", "ref_time_start"):
        setattr(b, n, e.v(n))
    if e.key in ("multipole", "ab_multipole"):
        _, knl, tn = L.multipole_ele_to_kt(e, True)
        b.knl[:] = list(knl)
        b.tn[:] = list(tn)
    else:
        _, a, bb = L.multipole_ele_to_ab(e, False, False, True)
        b.an[:] = list(a)
        b.bn[:] = list(bb)
        _, ae, be = L.multipole_ele_to_ab(e, False, True, False)
        b.an_elec[:] = list(ae)
        b.bn_elec[:] = list(be)
    return b


def element_key(e: L.Element) -> tuple:
    """Everything to_bgt_element reads from an element: equal keys give equal
    C structs (used to convert each distinct element of a variant family
    once)."""
    return (e.key, e.ix_ele, e.is_on, e.num_steps, e.fringe_type, e.fringe_at, e.aperture_type, e.aperture_at,
            e.offset_moves_aperture, e.exact_multipoles, e.scale_multipoles, e.has_misalign,
            tuple(sorted(e.values.items())), tuple(sorted(e.a_pole.items())), tuple(sorted(e.b_pole.items())),
            tuple(sorted(e.ksl_pole.items())), tuple(sorted(e.a_pole_elec.items())),
            tuple(sorted(e.b_pole_elec.items())))


def ptr(a: np.ndarray, t):
    return a.ctypes.data_as(C.POINTER(t))
