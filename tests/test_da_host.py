"""Host logic of the dynamic-aperture driver (bgt.da), on the CPU: the grid
and reference-orbit formulas of dynamic_aperture_scan
(bmad/modules/dynamic_aperture_mod.f90:88-95,132-136), the DA radius rule,
per-variant optics through a batched one-turn map (here the oracle), and the
lattice-error summary."""
from __future__ import annotations

import math

import numpy as np
import pytest

from bgt import da, optics, rings

from helpers import oracle_batch_one_turn


def test_ray_angles_and_radii():
    a = da.ray_angles(5, 0.0, math.pi)
    assert np.allclose(a, [0, math.pi / 4, math.pi / 2, 3 * math.pi / 4, math.pi], rtol=0, atol=1e-15)
    assert da.ray_angles(1, 0.2, 0.6)[0] == pytest.approx(0.4)
    r = da.grid_radii(64, 0.025)
    assert r[0] == 0 and r[-1] == pytest.approx(0.025) and len(r) == 64


def test_radius_from_survival():
    n_turns = 100
    s = np.full((2, 3, 8), n_turns, np.int32)
    s[0, 0, 5] = 40          # first loss at index 5 -> radius index 4
    s[0, 1, 0] = 0           # first point lost -> 0
    s[1, 2, 3:] = 7          # loss from index 3 -> index 2
    s[1, 0, 7] = 99          # last point lost on the last turn -> index 6
    r = da.radius_from_survival(s, n_turns, 0.007)
    dr = 0.007 / 7
    assert r[0, 0] == dr * 4 and r[0, 1] == 0.0 and r[0, 2] == dr * 7
    assert r[1, 2] == dr * 2 and r[1, 0] == dr * 6


def test_grid_initial_conditions_order_and_formula():
    ref = np.arange(2 * 3 * 6, dtype=np.float64).reshape(2, 3, 6) * 1e-4
    v6 = da.grid_initial_conditions(ref, 4, 0.0, math.pi, 5, 0.02, 0.6)
    assert v6.shape == (6, 2 * 3 * 4 * 5)
    ang = da.ray_angles(4, 0.0, math.pi)
    rad = da.grid_radii(5, 0.02)
    i = 0
    for v in range(2):
        for d in range(3):
            for a in range(4):
                for k in range(5):
                    exp = ref[v, d].copy()
                    exp[0] = exp[0] + math.cos(ang[a]) * rad[k]
                    exp[2] = exp[2] + (math.sin(ang[a]) * rad[k]) * 0.6
                    assert np.array_equal(v6[:, i], exp)
                    i += 1


def test_reference_orbits_add_dispersion():
    o = da.VariantOptics(np.ones((2, 6)) * 1e-5, np.array([[0.8, 0.1, 0.0, 0.0]] * 2), *(np.ones(2) for _ in range(6)))
    ref = da.reference_orbits(o, (-0.01, 0.0, 0.01))
    assert ref.shape == (2, 3, 6)
    assert ref[0, 0, 0] == pytest.approx(1e-5 - 0.008)
    assert ref[1, 2, 5] == pytest.approx(1e-5 + 0.01)
    assert np.array_equal(ref[:, 1], o.closed_orbit)


def test_variant_optics_matches_single_lattice_optics():
    lats = rings.error_variants(2, seed=7)
    f = oracle_batch_one_turn(lats)
    vo = da.variant_optics(f, 2)
    for v in range(2):
        one = lambda x, v=v: f(x, np.full(x.shape[1], v, np.int32))  # noqa: E731
        co = optics.closed_orbit(one, six_d=True)
        assert np.allclose(vo.closed_orbit[v], co, rtol=0, atol=1e-11)
    # misaligned quads give a closed-orbit distortion; tunes near the design
    assert np.max(np.abs(vo.closed_orbit[:, 0])) > 1e-7
    assert np.allclose(vo.tune_a, rings.TUNES0[0], atol=0.02) and np.allclose(vo.tune_b, rings.TUNES0[1], atol=0.02)
    assert np.allclose(vo.beta_a, rings.TWISS0["beta_a"], rtol=0.05)
    assert np.allclose(vo.eta[:, 0], rings.TWISS0["eta_x"], rtol=0.05)


def test_error_summary_scales():
    base = rings.fodo_ring(apertures=True)
    errs = rings.error_variants(3, seed=11)
    sx = rings.sextupole_variants(2, seed=5)
    s0 = da.error_summary([base], (rings.K2_SF, rings.K2_SD))
    assert s0.shape == (1, 16) and np.allclose(s0, 0)
    se = da.error_summary(errs, (rings.K2_SF, rings.K2_SD))
    assert np.all(se[:, :14] > 0.3) and np.all(se[:, :14] < 3.0) and np.allclose(se[:, 14:], 0)
    ss = da.error_summary(sx, (rings.K2_SF, rings.K2_SD))
    assert np.allclose(ss[:, :14], 0) and np.all(np.abs(ss[:, 14:]) <= 1.0 + 1e-12)


def test_ranking_mismatches():
    from bgt import learned_da as LD

    a = np.array([5.0, 4.0, 3.0, 2.0, 1.0])
    r = LD.ranking_mismatches(a, a.copy())
    assert r["discordant_pairs"] == 0 and r["spearman"] == pytest.approx(1.0) and r["pairs"] == 10
    b = np.array([4.0, 5.0, 3.0, 1.0, 2.0])  # two adjacent swaps
    r = LD.ranking_mismatches(a, b)
    assert r["discordant_pairs"] == 2 and r["rank_position_mismatches"] == 4
    r = LD.ranking_mismatches(a, a[::-1].copy())
    assert r["discordant_pairs"] == 10 and r["spearman"] == pytest.approx(-1.0)


def test_radius_of_survive_labels():
    from bgt import learned_da as LD

    class P:
        deltas = (0.0, 0.01)
        n_angle = 2
        n_radius = 5
        r_max = 0.004

    lab = np.ones((1, 2, 2, 5), bool)
    lab[0, 0, 1, 3] = False
    lab[0, 1, 0, 0] = False
    r = LD.radius_of(P, lab.reshape(-1), 1)
    assert r.shape == (1, 2, 2)
    assert r[0, 0, 0] == 0.004 and r[0, 0, 1] == 0.002 and r[0, 1, 0] == 0.0 and r[0, 1, 1] == 0.004
