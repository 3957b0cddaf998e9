"""Dynamic-aperture pieces on the GPU against the correctly rounded oracle:
device tracking with per-particle variants, per-variant optics through the
GPU one-turn map, and the one-launch polar-grid scan of error variants
(bgt.da), all bit-identical."""
from __future__ import annotations

import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from helpers import oracle_batch_one_turn, oracle_da_survival  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def variants():
    from bgt import rings

    return rings.error_variants(3, seed=21)


def test_device_variants_equal_host_variants(variants):
    from bgt import lattice as L
    from bgt import rings
    from bgt.track import Tracker

    tr = Tracker(variants)
    n = 3000
    v0 = rings.gaussian_beam(rings.CONFIG1_BEAM, n=n)
    var = np.sort(np.random.default_rng(1).integers(0, 3, n)).astype(np.int32)
    hb = tr.make_bunch(v0.copy())
    tr.track_turns(hb, 7, variant=var)
    dev = torch.device("cuda", 0)
    vec = torch.tensor(v0, device=dev).contiguous()
    beta = torch.tensor(L.beta_of(tr.p0c, v0[5], tr.species.mass), device=dev)
    st = torch.ones(n, dtype=torch.int32, device=dev)
    ie = torch.full((n,), -1, dtype=torch.int32, device=dev)
    it = torch.full((n,), -1, dtype=torch.int32, device=dev)
    tr.track_turns_device(vec, beta, st, ie, it, 7, variant=torch.tensor(var, device=dev))
    torch.cuda.synchronize()
    assert np.array_equal(vec.cpu().numpy(), hb.vec6)
    assert np.array_equal(st.cpu().numpy(), hb.state)
    assert np.array_equal(it.cpu().numpy(), hb.ix_turn_lost)


def test_device_variants_must_be_sorted(variants):
    from bgt import _lib
    from bgt.track import Tracker

    tr = Tracker(variants)
    dev = torch.device("cuda", 0)
    n = 256
    vec = torch.zeros(6, n, dtype=torch.float64, device=dev)
    beta = torch.full((n,), 0.999, dtype=torch.float64, device=dev)
    st = torch.ones(n, dtype=torch.int32, device=dev)
    ie = torch.full((n,), -1, dtype=torch.int32, device=dev)
    it = torch.full((n,), -1, dtype=torch.int32, device=dev)
    var = torch.tensor(np.r_[np.ones(128), np.zeros(128)].astype(np.int32), device=dev)
    with pytest.raises(_lib.BgtError, match="sorted"):
        tr.track_turns_device(vec, beta, st, ie, it, 1, variant=var)


def test_variant_optics_gpu_equals_oracle(variants):
    from bgt import da
    from bgt.track import Tracker

    tr = Tracker(variants)
    g = da.variant_optics(da.tracker_one_turn(tr), 3)
    o = da.variant_optics(oracle_batch_one_turn(variants, variant="cr"), 3)
    assert np.array_equal(g.closed_orbit, o.closed_orbit)
    assert np.array_equal(g.eta, o.eta)
    assert np.array_equal(g.beta_a, o.beta_a) and np.array_equal(g.tune_b, o.tune_b)


def test_plain_scan_equals_oracle(variants):
    from bgt import da
    from bgt.track import Tracker

    tr = Tracker(variants)
    opt = da.variant_optics(da.tracker_one_turn(tr), 3)
    ref = da.reference_orbits(opt, (-0.01, 0.0, 0.01))
    ys = da.y_scale(opt.beta_a[0], opt.beta_b[0])
    grid = dict(n_angle=5, angle_min=0.0, angle_max=math.pi, n_radius=12, r_max=0.03, yscale=ys)
    res = da.plain_scan(tr, ref, n_turns=40, **grid)
    surv = oracle_da_survival(variants, ref, n_turns=40, **grid)
    assert np.array_equal(res.survive_turns, surv)
    assert np.array_equal(res.radius, da.radius_from_survival(surv, 40, 0.03))
    assert np.any(res.radius < 0.03) and np.any(res.radius > 0)


def _two_error_rings():
    """Two error variants' element lists in one ring: ~1540 elements, ~300 KB
    of distinct element records -- more than one CTA's shared memory."""
    import copy

    from bgt import lattice as L
    from bgt import rings

    a, b = rings.error_variants(2, seed=33)
    els = [copy.deepcopy(e) for e in a.elements[:-2]] + [copy.deepcopy(e) for e in b.elements]
    return L.Lattice(els, a.species, a.p0c, a.e_tot, "two_error_rings").finalize()


@pytest.mark.parametrize("mode", ["auto", "global", "global-warp"])
def test_large_table_global_memory_path(mode):
    """Element tables too large for shared memory are read from global memory
    (table_mode 0 picks it, 2 forces it, 3 with per-warp scheduling); results
    stay bit-identical to the correctly rounded oracle, and table_mode 1
    refuses such a table."""
    from bgt import _lib, rings
    from bgt.track import Tracker
    from helpers import oracle_track_elements

    lat = _two_error_rings()
    tr = Tracker(lat)
    assert tr.table_bytes() > 224 * 1024
    tr.set_tuning(threads_per_block=256, blocks_per_sm=2, table_mode={"auto": 0, "global": 2, "global-warp": 3}[mode])
    v0 = rings.gaussian_beam(rings.CONFIG1_BEAM, n=1024)
    b = tr.make_bunch(v0.copy())
    tr.track_turns(b, 3)
    ov, _, ost, oie, _ = oracle_track_elements(lat, v0.copy(), 0, len(lat), n_turns=3, variant="cr")
    assert np.array_equal(b.vec6, ov) and np.array_equal(b.state, ost) and np.array_equal(b.ix_ele_lost, oie)
    tr.set_tuning(threads_per_block=256, blocks_per_sm=2, table_mode=1)
    with pytest.raises(_lib.BgtError, match="shared memory"):
        tr.track_turns(tr.make_bunch(v0.copy()), 1)


def test_error_variant_ring_matches_oracle():
    """A full error-variant ring (every quadrupole with 16 kick-drift steps
    and multipoles b3..b6 / a3..a6, offsets and rolls) over 20 turns:
    bit-identical to the correctly rounded oracle, in every table mode."""
    from bgt import rings
    from bgt.track import Tracker
    from helpers import oracle_track_elements

    lat = rings.error_variants(1, seed=44)[0]
    v0 = rings.gaussian_beam(rings.CONFIG1_BEAM, n=2048)
    ov, _, ost, oie, oit = oracle_track_elements(lat, v0.copy(), 0, len(lat), n_turns=20, variant="cr")
    tr = Tracker(lat)
    for mode in (1, 2, 3):
        tr.set_tuning(threads_per_block=128, blocks_per_sm=4, table_mode=mode)
        b = tr.make_bunch(v0.copy())
        tr.track_turns(b, 20)
        assert np.array_equal(b.vec6, ov) and np.array_equal(b.state, ost)
        assert np.array_equal(b.ix_ele_lost, oie) and np.array_equal(b.ix_turn_lost, oit)


def test_staged_scan_equals_one_launch_scan(variants):
    """The Python driver's two-launch scan (turn-64 snapshot, radius-major
    tracking order) gives the one-launch scan's survival turns exactly."""
    from bgt import da, rings
    from bgt import learned_da as LD
    from bgt.track import Tracker

    grid = rings.DAGrid(6, 16, 0.03, (-0.01, 0.0), 90)
    pb = LD.setup(Tracker(variants), variants, grid)
    st = LD.staged_scan(pb, 0, 3, early=20)
    plain = da.plain_scan(pb.tracker, pb.ref, **pb.grid())
    assert np.array_equal(st.survive.cpu().numpy(), plain.survive_turns.reshape(-1))
    assert np.any(plain.survive_turns < 90) and np.any(plain.survive_turns == 90)


@pytest.mark.parametrize("retune", [False, True])
def test_compacted_scan_equals_one_launch_scan(variants, retune):
    """The compacted plain scan (every probe 5 turns, then the live probes
    packed densely, optionally with a re-tuned launch shape) gives the
    one-launch scan's survival turns, radii and particle.turns exactly, with
    losses in both launches."""
    from bgt import da, rings
    from bgt import learned_da as LD
    from bgt.track import Tracker

    grid = rings.DAGrid(6, 16, 0.03, (-0.01, 0.0), 90)
    pb = LD.setup(Tracker(variants), variants, grid)
    tun = pb.tracker.get_tuning()
    cs = LD.compacted_scan(pb, 0, 3, early=5, retune_subset=retune)
    assert pb.tracker.get_tuning() == tun  # the scan's tuning is restored
    plain = da.plain_scan(pb.tracker, pb.ref, **pb.grid())
    assert np.array_equal(cs.survive_turns, plain.survive_turns)
    assert np.array_equal(cs.radius, plain.radius)
    assert cs.particle_turns == plain.particle_turns
    s = plain.survive_turns
    assert np.any(s < 5) and np.any((s >= 5) & (s < 90)) and np.any(s == 90)
