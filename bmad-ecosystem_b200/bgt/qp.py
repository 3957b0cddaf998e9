"""Particle times as IEEE binary128 values (the reference's real(qp)
coord_struct%t) held in numpy: an (n, 2) uint64 array, word 0 the low 64
bits and word 1 the high 64 bits -- the memory layout of a C __float128 or a
Fortran real(qp) array on x86-64, which the C ABI takes as it is.

Only the conversions the host needs: a double to binary128 (exact, as a
Fortran real(qp) assignment of a real(rp) value) and binary128 to the nearest
double (ties to even), vectorised.
"""
from __future__ import annotations

import numpy as np

_M52 = np.uint64((1 << 52) - 1)
_M48 = np.uint64((1 << 48) - 1)
_NAN_HI = np.uint64(0x7FFF800000000000)


def from_double(x) -> np.ndarray:
    """Exact binary128 bits of float64 values: (n, 2) uint64."""
    x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
    b = x.view(np.uint64)
    sign = b >> np.uint64(63)
    ex = ((b >> np.uint64(52)) & np.uint64(0x7FF)).astype(np.int64)
    fr = b & _M52
    out = np.zeros((x.size, 2), dtype=np.uint64)
    normal = (ex > 0) & (ex < 0x7FF)
    e = (ex + (16383 - 1023)).astype(np.uint64)
    out[normal, 0] = fr[normal] << np.uint64(60)
    out[normal, 1] = (sign[normal] << np.uint64(63)) | (e[normal] << np.uint64(48)) | (fr[normal] >> np.uint64(4))
    zero = (ex == 0) & (fr == 0)
    out[zero, 1] = sign[zero] << np.uint64(63)
    out[ex == 0x7FF, 1] = _NAN_HI
    for i in np.nonzero((ex == 0) & (fr != 0))[0]:  # subnormal doubles: normalised
        f = int(fr[i])
        lz = 52 - (f.bit_length() - 1)
        f = (f << lz) & ((1 << 52) - 1)
        eb = -1022 - lz + 16383
        out[i, 0] = np.uint64((f << 60) & ((1 << 64) - 1))
        out[i, 1] = np.uint64((int(sign[i]) << 63) | (eb << 48) | (f >> 4))
    return out


def to_double(q) -> np.ndarray:
    """Nearest float64 (ties to even) of binary128 bits, (n, 2) uint64, for
    values in the normal double range or zero; NaN for NaN or infinity."""
    q = np.ascontiguousarray(q, dtype=np.uint64).reshape(-1, 2)
    lo, hi = q[:, 0], q[:, 1]
    sign = hi >> np.uint64(63)
    ebits = ((hi >> np.uint64(48)) & np.uint64(0x7FFF)).astype(np.int64)
    k = (((hi & _M48) | np.uint64(1 << 48)) << np.uint64(4)) | (lo >> np.uint64(60))  # 53 bits
    rest = lo & np.uint64((1 << 60) - 1)
    half = np.uint64(1 << 59)
    up = (rest > half) | ((rest == half) & ((k & np.uint64(1)) == np.uint64(1)))
    k = k + up.astype(np.uint64)
    e = ebits - 16383
    carry = (k >> np.uint64(53)) != 0
    k = np.where(carry, k >> np.uint64(1), k)
    e = np.where(carry, e + 1, e)
    bits = (sign << np.uint64(63)) | ((e + 1023).astype(np.uint64) << np.uint64(52)) | (k & _M52)
    zero = (ebits == 0) & ((hi & _M48) == 0) & (lo == 0)
    bits = np.where(zero, sign << np.uint64(63), bits)
    out = bits.view(np.float64).copy()
    out[ebits == 0x7FFF] = np.nan
    return out


def initial_time(vec6: np.ndarray, beta: np.ndarray, ref_time: float = 0.0) -> np.ndarray:
    """init_coord's particle time t = ref_time - z / (beta c_light)
    (bmad/low_level/init_coord.f90:222), evaluated in real(rp), as binary128."""
    from .lattice import C_LIGHT

    z = np.asarray(vec6, dtype=np.float64)[4]
    return from_double(ref_time - z / (np.asarray(beta, dtype=np.float64) * C_LIGHT))
