"""GPU parity: the CUDA tracker (through the C ABI) against the CPU oracle on
identical seeded particles.

Two oracle builds are used:
* "cr"    -- transcendentals of particle coordinates correctly rounded, the
             device's own contract: results must be bit-identical.
* "glibc" -- transcendentals from the C library, as the reference evaluates
             them.  glibc 2.39 is correctly rounded on all but ~0.01-0.2% of
             the sin/asin/atan2 arguments, so results agree to within
             RTOL_ONE_TURN = 1e-13 relative per coordinate after one turn and
             RTOL_1000_TURNS = 1e-9 after 1000 turns (tests/helpers.py), with
             states, loss elements and loss turns exact.
"""
import numpy as np
import pytest

from bgt import lattice as L
from bgt import rings
from bgt.track import Bunch, Tracker

from helpers import (RTOL_1000_TURNS, RTOL_LIBM_1000_TURNS, RTOL_LIBM_ONE_TURN, RTOL_ONE_TURN,
                     oracle_track_elements, random_particles, rare_zoo_lattice, rel_err, rtol_vs_glibc_one_element,
                     zoo_lattice)

pytestmark = pytest.mark.gpu


def assert_bitwise(b, ov, ob, ost, oie, oit=None, what=""):
    assert np.array_equal(b.state, ost), f"{what}: state"
    assert np.array_equal(b.ix_ele_lost, oie), f"{what}: loss element"
    if oit is not None:
        assert np.array_equal(b.ix_turn_lost, oit), f"{what}: loss turn"
    assert np.array_equal(b.vec6, ov), f"{what}: coordinates differ (max abs {np.max(np.abs(b.vec6 - ov))})"
    assert np.array_equal(b.beta, ob), f"{what}: beta"


@pytest.fixture(scope="module")
def zoo():
    lat = zoo_lattice()
    return lat, Tracker(lat)


def test_each_element_track1_bitwise(zoo):
    lat, tr = zoo
    v0 = random_particles(2048, seed=11)
    for pos, ele in enumerate(lat.elements):
        b = tr.make_bunch(v0.copy())
        tr.track1(b, pos)
        ov, ob, ost, oie, _ = oracle_track_elements(lat, v0, pos, pos + 1, variant="cr")
        assert_bitwise(b, ov, ob, ost, oie, what=ele.name)


def test_each_element_track1_vs_glibc(zoo):
    lat, tr = zoo
    v0 = random_particles(2048, seed=11)
    for pos, ele in enumerate(lat.elements):
        b = tr.make_bunch(v0.copy())
        tr.track1(b, pos)
        ov, ob, ost, oie, _ = oracle_track_elements(lat, v0, pos, pos + 1)
        assert np.array_equal(b.state, ost), f"{ele.name}: state mismatch"
        alive = ost == L.ALIVE
        err = rel_err(b.vec6, ov, alive)
        assert np.all(err <= RTOL_ONE_TURN), f"{ele.name}: rel err {err}"


def test_zoo_pass_with_losses(zoo):
    lat, tr = zoo
    v0 = random_particles(4096, seed=12, scale=4.0)
    b = tr.make_bunch(v0.copy())
    tr.track_elements(b, 0, len(lat))
    ov, ob, ost, oie, _ = oracle_track_elements(lat, v0, 0, len(lat), variant="cr")
    assert (ost != L.ALIVE).sum() > 100  # the case exercises losses
    assert_bitwise(b, ov, ob, ost, oie, what="zoo pass")


@pytest.fixture(scope="module")
def rare_zoo():
    lat = rare_zoo_lattice()
    return lat, Tracker(lat)


def test_rare_zoo_each_element_bitwise(rare_zoo):
    # misaligned and electric bends, electric quadrupoles, edge fringe and
    # element-frame apertures: the RARE kernels against the oracle
    lat, tr = rare_zoo
    v0 = random_particles(2048, seed=21)
    for pos, ele in enumerate(lat.elements):
        b = tr.make_bunch(v0.copy())
        tr.track1(b, pos)
        ov, ob, ost, oie, _ = oracle_track_elements(lat, v0, pos, pos + 1, variant="cr")
        assert_bitwise(b, ov, ob, ost, oie, what=ele.name)
        ovg, _, ostg, _, _ = oracle_track_elements(lat, v0, pos, pos + 1)
        assert np.array_equal(b.state, ostg), f"{ele.name}: state vs glibc oracle"
        assert np.all(rel_err(b.vec6, ovg, ostg == L.ALIVE) <= rtol_vs_glibc_one_element(ele)), ele.name


def test_rare_zoo_turns_with_losses(rare_zoo):
    lat, tr = rare_zoo
    # the line does not close, so the orbit grows turn by turn: particles are
    # lost at the collimators over all five turns
    v0 = random_particles(4096, seed=22, scale=0.1)
    b = tr.make_bunch(v0.copy())
    tr.track_turns(b, 5)
    ov, ob, ost, oie, oit = oracle_track_elements(lat, v0, 0, len(lat), 5, variant="cr")
    assert len(np.unique(oit[ost != L.ALIVE])) == 5 and (ost == L.ALIVE).sum() > 0
    assert_bitwise(b, ov, ob, ost, oie, oit, what="rare zoo, 5 turns")


@pytest.fixture(scope="module")
def ring():
    lat = rings.fodo_ring()
    return lat, Tracker(lat)


def test_ring_one_turn(ring):
    lat, tr = ring
    v0 = rings.gaussian_beam(rings.CONFIG0_BEAM)
    b = tr.make_bunch(v0.copy())
    tr.track_turns(b, 1)
    ov, ob, ost, oie, oit = oracle_track_elements(lat, v0, 0, len(lat), 1, variant="cr")
    assert_bitwise(b, ov, ob, ost, oie, oit, "one turn vs cr")
    gv, gb, gst, _, _ = oracle_track_elements(lat, v0, 0, len(lat), 1)
    assert np.all(gst == L.ALIVE)
    err = rel_err(b.vec6, gv)
    assert np.all(err <= RTOL_LIBM_ONE_TURN), err
    # most particles see no glibc rounding difference in one turn: those are
    # within RTOL_ONE_TURN (in fact identical)
    per = np.max(np.abs(b.vec6 - gv) / (np.abs(gv) + np.sqrt(np.mean(gv * gv, axis=1))[:, None]), axis=0)
    assert np.mean(per <= RTOL_ONE_TURN) > 0.5


def test_ring_1000_turns(ring):
    lat, tr = ring
    v0 = rings.gaussian_beam(rings.CONFIG0_BEAM, n=1000)
    b = tr.make_bunch(v0.copy())
    tr.track_turns(b, 1000)
    ov, ob, ost, oie, oit = oracle_track_elements(lat, v0, 0, len(lat), 1000, variant="cr")
    assert_bitwise(b, ov, ob, ost, oie, oit, "1000 turns vs cr")
    gv, gb, gst, _, _ = oracle_track_elements(lat, v0, 0, len(lat), 1000)
    assert np.all(gst == L.ALIVE) and np.all(b.state == L.ALIVE)
    err = rel_err(b.vec6, gv)
    assert np.all(err <= RTOL_LIBM_1000_TURNS), err


def test_apertures_loss_records():
    lat = rings.fodo_ring(apertures=True)
    tr = Tracker(lat)
    # a beam large enough to scrape the 20 mm x 10 mm quad apertures
    spec = rings.BeamSpec(3000, 4e-6, 2e-6, 3e-3, 2e-3, seed=77)
    v0 = rings.gaussian_beam(spec)
    b = tr.make_bunch(v0.copy())
    tr.track_turns(b, 50)
    ov, ob, ost, oie, oit = oracle_track_elements(lat, v0, 0, len(lat), 50, variant="cr")
    assert int((ost != L.ALIVE).sum()) > 50
    assert_bitwise(b, ov, ob, ost, oie, oit, "apertures vs cr")
    # against the C-library oracle: loss element and turn exact for every
    # particle (none of these pass within 1e-9 m of an edge undetected)
    gv, gb, gst, gie, git = oracle_track_elements(lat, v0, 0, len(lat), 50)
    assert np.array_equal(b.state, gst)
    assert np.array_equal(b.ix_ele_lost, gie)
    assert np.array_equal(b.ix_turn_lost, git)


def test_compaction_and_tiles_do_not_change_results():
    lat = rings.fodo_ring(apertures=True)
    spec = rings.BeamSpec(5000, 4e-6, 2e-6, 3e-3, 2e-3, seed=78)
    v0 = rings.gaussian_beam(spec)
    outs = []
    for tun in (dict(threads_per_block=128, blocks_per_sm=4),
                dict(threads_per_block=64, blocks_per_sm=8, compact_every=2, turns_per_launch=7),
                dict(threads_per_block=256, blocks_per_sm=2, compact_every=1)):
        tr = Tracker(lat, tuning=tun)
        b = tr.make_bunch(v0.copy())
        tr.track_turns(b, 30)
        outs.append(b)
    for o in outs[1:]:
        assert np.array_equal(o.state, outs[0].state)
        assert np.array_equal(o.ix_ele_lost, outs[0].ix_ele_lost)
        assert np.array_equal(o.ix_turn_lost, outs[0].ix_turn_lost)
        assert np.array_equal(o.vec6, outs[0].vec6)


def test_ragged_sizes_empty_calls_and_lost_input():
    """Particle counts that fill no tile (1, 33, 257) in every table
    placement, a nonzero start turn (loss turns are absolute), the empty
    call, zero turns, and particles already lost on input (left as they
    are)."""
    lat = rings.fodo_ring(apertures=True)
    v_all = rings.gaussian_beam(rings.BeamSpec(300, 4e-6, 2e-6, 3e-3, 2e-3, seed=79))
    for mode in (0, 2, 3):
        tr = Tracker(lat, tuning=dict(threads_per_block=128, blocks_per_sm=4, table_mode=mode))
        for n in (1, 33, 257):
            v0 = v_all[:, :n].copy()
            b = tr.make_bunch(v0.copy())
            tr.track_turns(b, 20, turn0=5)
            ov, ob, ost, oie, oit = oracle_track_elements(lat, v0, 0, len(lat), 20, variant="cr")
            oit = np.where(ost != L.ALIVE, oit + 5, oit)
            assert_bitwise(b, ov, ob, ost, oie, oit, f"n={n} table_mode={mode}")
    tr = Tracker(lat)
    launches = tr.launch_count
    empty = tr.make_bunch(np.zeros((6, 0)))
    tr.track_turns(empty, 5)
    b = tr.make_bunch(v_all.copy())
    tr.track_turns(b, 0)
    assert tr.launch_count == launches and np.array_equal(b.vec6, v_all)
    b.state[::3] = L.LOST_NEG_X
    b.ix_ele_lost[::3] = 7
    b.ix_turn_lost[::3] = 2
    before = b.vec6[:, ::3].copy()
    tr.track_turns(b, 10, turn0=3)
    assert np.array_equal(b.vec6[:, ::3], before)
    assert np.all(b.state[::3] == L.LOST_NEG_X) and np.all(b.ix_ele_lost[::3] == 7)
    assert np.all(b.ix_turn_lost[::3] == 2)


def test_variants_batched():
    lats = rings.error_variants(4, seed=5)
    tr = Tracker(lats)
    n = 1200
    v0 = random_particles(n, seed=13, scale=0.5)
    var = np.arange(n, dtype=np.int32) % 4
    b = tr.make_bunch(v0.copy())
    tr.track_turns(b, 3, variant=var)
    for v in range(4):
        m = var == v
        ov, ob, ost, oie, oit = oracle_track_elements(lats[v], v0[:, m], 0, len(lats[v]), 3, variant="cr")
        assert np.array_equal(b.state[m], ost)
        assert np.array_equal(b.ix_ele_lost[m], oie)
        assert np.array_equal(b.vec6[:, m], ov), (v, np.max(np.abs(b.vec6[:, m] - ov)))


def test_device_api_matches_host_api(ring):
    import torch

    lat, tr = ring
    v0 = rings.gaussian_beam(rings.CONFIG0_BEAM, n=4096)
    b = tr.make_bunch(v0.copy())
    tr.track_turns(b, 5)
    dv = torch.tensor(v0, dtype=torch.float64, device="cuda").contiguous()
    db = torch.tensor(L.beta_of(lat.p0c, v0[5], lat.species.mass), device="cuda")
    ds = torch.ones(4096, dtype=torch.int32, device="cuda")
    de = torch.full((4096,), -1, dtype=torch.int32, device="cuda")
    dt = torch.full((4096,), -1, dtype=torch.int32, device="cuda")
    tr.track_turns_device(dv, db, ds, de, dt, 5)
    torch.cuda.synchronize()
    assert np.array_equal(dv.cpu().numpy(), b.vec6)
    assert np.array_equal(ds.cpu().numpy(), b.state)


def test_da_grid_matches_oracle():
    import math

    lat = rings.fodo_ring(apertures=True)
    tr = Tracker(lat)
    ref = np.zeros((1, 2, 6))
    ref[0, 1, 5] = 0.005
    ref[0, 1, 0] = 0.005 * rings.TWISS0["eta_x"]
    ref[0, 1, 1] = 0.005 * rings.TWISS0["etap_x"]
    n_angle, n_radius, r_max, turns = 6, 12, 0.03, 40
    da, surv = tr.da_scan_grid(ref, n_angle, 0.0, np.pi, n_radius, r_max, 1.0, turns, return_survival=True)
    dang = (np.pi - 0.0) / (n_angle - 1)
    dr = r_max / (n_radius - 1)
    for d in range(2):
        pts = []
        for ia in range(n_angle):
            ang = ia * dang + 0.0  # dynamic_aperture_mod.f90:88-95
            for ir in range(n_radius):
                rad = dr * ir
                p = ref[0, d].copy()
                p[0] = p[0] + math.cos(ang) * rad
                p[2] = p[2] + math.sin(ang) * rad * 1.0
                pts.append(p)
        v0 = np.array(pts).T.copy()
        ov, ob, ost, oie, oit = oracle_track_elements(lat, v0, 0, len(lat), turns, variant="cr")
        s = np.where(ost == L.ALIVE, turns, oit)
        assert np.array_equal(surv[0, d].reshape(-1), s)
        alive = (ost == L.ALIVE).reshape(n_angle, n_radius)
        for ia in range(n_angle):
            lost = np.nonzero(~alive[ia])[0]
            first = lost[0] if lost.size else n_radius
            expect = 0.0 if first == 0 else dr * (first - 1)
            assert da[0, d, ia] == expect
