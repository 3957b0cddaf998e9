"""The device's correctly rounded transcendentals (sin, cos, sinh, cosh, exp,
asin, atan2), compiled for the host.

bgt_crmath.cuh is host/device code.  Here it is compiled with g++ (no FMA
contraction, like the device build's --fmad=false) into tests/crmath_check.cpp
and every result is compared with libquadmath evaluated in binary128 and
rounded to double: the light small-argument paths, the double-double fast
paths and the slow paths behind them must all return the correctly rounded
double.  A larger sample of the same program (millions per range) is run
whenever the paths change.
"""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "crmath_check.cpp"


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = tmp_path_factory.mktemp("crmath") / "crmath_check"
    subprocess.run([gxx, "-O2", "-ffp-contract=off", "-std=c++17", "-o", str(exe), str(SRC), "-lquadmath"],
                   check=True, capture_output=True)
    return exe


@pytest.mark.parametrize("seed", [1, 2])
def test_correctly_rounded_against_binary128(checker, seed):
    r = subprocess.run([str(checker), "40000", str(seed)], capture_output=True, text=True, timeout=600)
    lines = [ln.split() for ln in r.stdout.splitlines() if ln and not ln.startswith("MISMATCH")]
    assert len(lines) >= 21
    bad = {f"{fn}[{lo},{hi}]": int(nb) for fn, lo, hi, nb, n in lines if int(nb)}
    assert r.returncode == 0 and not bad, r.stdout

