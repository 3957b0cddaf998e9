"""The roofline numerator: bench.py's FP64 operations and libm calls per
particle.turn of the config-1 workload are what the instrumented oracle
build counts on the config-1 ring and beam (add/sub/mul/div/sqrt = 1 each;
libm calls separately).  The count depends only on the branches the
particles take, so a sample of the beam gives the same figure."""
import importlib.util
from pathlib import Path

import pytest

from bgt import rings

ROOT = Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", ROOT / "bench.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_bench_constants_match_the_counted_oracle(oracle_lib):
    from oracle import oracle as O

    b = _bench()
    lat = rings.fodo_ring(apertures=True)
    v = rings.gaussian_beam(rings.CONFIG1_BEAM, n=2000)
    flops, libm = O.flops_per_particle_turn(lat, v, n_turns=2)
    assert flops == pytest.approx(b.FLOPS_PER_PARTICLE_TURN, rel=1e-9)
    assert libm == pytest.approx(b.LIBM_PER_PARTICLE_TURN, rel=1e-9)


def test_error_ring_count(oracle_lib):
    """The config-2 error ring's count quoted beside the DA-scan numbers:
    16-step quadrupoles with order-6 kicks, offsets and rolls."""
    from oracle import oracle as O

    lat = rings.error_variants(1, seed=3)[0]
    v = rings.gaussian_beam(rings.CONFIG1_BEAM, n=200)
    flops, libm = O.flops_per_particle_turn(lat, v)
    assert flops == pytest.approx(902_775.0, rel=1e-9)
    assert libm == pytest.approx(11_019.0, rel=1e-9)
