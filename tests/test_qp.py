"""The software binary128 arithmetic the device uses for the particle time
(bmad-ecosystem_b200/csrc/bgt_qp.cuh), built for the host and checked bit
for bit against GCC's __float128 (libquadmath), and the host-side numpy
conversions of bgt.qp against the same."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_binary128_arithmetic_matches_libquadmath(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = tmp_path / "qp_check"
    subprocess.run([gxx, "-O2", "-std=c++17", "-o", str(exe), str(ROOT / "tests" / "qp_check.cpp"), "-lquadmath"],
                   check=True, capture_output=True)
    for seed in (7, 2026):
        r = subprocess.run([str(exe), "400000", str(seed)], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        assert r.stdout.startswith("mismatches 0 of ")


def test_numpy_conversions_round_trip():
    from bgt import qp

    rng = np.random.default_rng(5)
    x = np.concatenate([rng.standard_normal(20000) * 10.0 ** rng.integers(-300, 300, 20000),
                        [0.0, -0.0, 5e-324, -2.2e-308, 1.7e308, 1.0, -1.0]])
    q = qp.from_double(x)
    assert q.shape == (x.size, 2) and q.dtype == np.uint64
    # the exact value of every binary128 produced, subnormal doubles included
    from fractions import Fraction

    for xi, (lo, hi) in zip(x[-7:], q[-7:]):
        lo, hi = int(lo), int(hi)
        e = (hi >> 48) & 0x7FFF
        frac = ((hi & ((1 << 48) - 1)) << 64) | lo
        val = Fraction(0) if e == 0 else (1 + Fraction(frac, 1 << 112)) * Fraction(2) ** (e - 16383)
        assert (-val if hi >> 63 else val) == Fraction(float(xi)) and (hi >> 63) == int(np.signbit(xi))
    # to_double (normal range and zeros) inverts it exactly, signs of zeros included
    keep = (np.abs(x) >= np.finfo(np.float64).tiny) | (x == 0)
    back = qp.to_double(q[keep])
    assert np.array_equal(back.view(np.uint64), x[keep].view(np.uint64))
    # binary128 values between doubles round to the nearest, ties to even
    q2 = q.copy()
    q2[:, 0] |= np.uint64(1 << 59)  # exactly half an ulp of the double above x
    r = qp.to_double(q2[:-7])
    xs = x[:-7]
    assert np.all(np.abs(xs) >= np.finfo(np.float64).tiny)
    up = np.nextafter(xs, np.copysign(np.inf, xs))
    even = np.where((xs.view(np.uint64) & np.uint64(1)) == 0, xs, up)
    assert np.array_equal(r, even)
