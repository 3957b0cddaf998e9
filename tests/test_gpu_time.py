"""The particle time t on the GPU: binary128 arithmetic in software
(bgt_qp.cuh), advanced in every element as the reference advances its
real(qp) coord_struct%t, and -- with bmad_com%absolute_time_tracking = T, the
dynamic_aperture program's setting (bsim/dynamic_aperture/
dynamic_aperture.f90:54) -- the RF phase taken from it
(particle_rf_time.f90:74-76,116-118).  Checked bit for bit, coordinates and
time, against the oracle (quad-precision time, correctly rounded
transcendentals), through the host-buffer and device-buffer entry points
and the DA scan."""
import numpy as np
import pytest

from bgt import lattice as L
from bgt import rings
from bgt.track import Tracker

from helpers import oracle_track_timed, random_particles, zoo_lattice

pytestmark = pytest.mark.gpu


def _assert_same(b, ref, what):
    ov, ob, ost, oie, oit, ot = ref
    assert np.array_equal(b.state, ost), what
    assert np.array_equal(b.ix_ele_lost, oie), what
    assert np.array_equal(b.ix_turn_lost, oit), what
    assert np.array_equal(b.vec6, ov), what
    assert np.array_equal(b.beta, ob), what
    assert np.array_equal(b.t, ot), what


def test_ring_in_absolute_time_bitwise():
    lat = rings.fodo_ring(apertures=True)
    v0 = rings.gaussian_beam(rings.BeamSpec(3000, 4e-6, 2e-6, 3e-3, 2e-3, seed=601))
    tr = Tracker(lat, absolute_time=True)
    b = tr.make_bunch(v0.copy())
    assert b.t is not None
    tr.track_turns(b, 100)
    ref = oracle_track_timed(lat, v0, 0, len(lat), 100, absolute_time=True)
    assert (ref[2] != L.ALIVE).sum() > 10
    _assert_same(b, ref, "ring, absolute time, 100 turns")
    # the time grows by one revolution period a turn
    alive = b.state == L.ALIVE
    t_rev = sum(e.v("delta_ref_time") for e in lat.elements)
    assert np.allclose(b.time[alive] - tr.make_bunch(v0).time[alive], 100 * t_rev, rtol=1e-9)


def test_time_in_relative_mode_changes_no_coordinate():
    """Carrying t with relative RF time runs the kernel instances that track
    time; coordinates equal the lean instance's bit for bit and t the
    oracle's."""
    lat = zoo_lattice()
    tr = Tracker(lat)
    v0 = random_particles(2000, seed=602, scale=2.0)
    plain = tr.make_bunch(v0.copy())
    tr.track_turns(plain, 4)
    timed = tr.make_bunch(v0.copy(), with_time=True)
    tr.track_turns(timed, 4)
    assert np.array_equal(plain.vec6, timed.vec6) and np.array_equal(plain.state, timed.state)
    _assert_same(timed, oracle_track_timed(lat, v0, 0, len(lat), 4), "zoo, relative time")


def test_device_buffers_carry_time():
    import torch

    lat = rings.fodo_ring(apertures=True)
    v0 = rings.gaussian_beam(rings.BeamSpec(2500, 4e-6, 2e-6, 3e-3, 2e-3, seed=603))
    tr = Tracker(lat, absolute_time=True)
    hb = tr.make_bunch(v0.copy())
    t0 = hb.t.copy()
    tr.track_turns(hb, 30)
    n = v0.shape[1]
    dv = torch.tensor(v0, dtype=torch.float64, device="cuda").contiguous()
    db = torch.tensor(L.beta_of(lat.p0c, v0[5], lat.species.mass), device="cuda")
    dt = torch.tensor(t0.view(np.int64), device="cuda").contiguous()
    ds = torch.ones(n, dtype=torch.int32, device="cuda")
    de = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    di = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    with pytest.raises(Exception, match="particle times"):
        tr.track_turns_device(dv, db, ds, de, di, 30)  # absolute time needs t
    tr.track_turns_device(dv, db, ds, de, di, 30, t=dt)
    tr.device_status()
    assert np.array_equal(dv.cpu().numpy(), hb.vec6)
    assert np.array_equal(dt.cpu().numpy().view(np.uint64), hb.t)
    assert np.array_equal(di.cpu().numpy(), hb.ix_turn_lost)


def test_da_scan_in_absolute_time_matches_oracle():
    """The DA scan with absolute time tracking (each probe's t from
    init_coord at the scan's start) equals the oracle probe by probe."""
    import math

    lat = rings.fodo_ring(apertures=True)
    tr = Tracker(lat, absolute_time=True)
    ref = np.zeros((1, 2, 6))
    ref[0, 1, 5] = 0.004
    n_angle, n_radius, r_max, turns = 5, 10, 0.03, 30
    da, surv = tr.da_scan_grid(ref, n_angle, 0.0, math.pi, n_radius, r_max, 1.0, turns, return_survival=True)
    dang = math.pi / (n_angle - 1)
    dr = r_max / (n_radius - 1)
    for d in range(2):
        pts = []
        for ia in range(n_angle):
            for ir in range(n_radius):
                p = ref[0, d].copy()
                p[0] = p[0] + math.cos(ia * dang) * (dr * ir)
                p[2] = p[2] + math.sin(ia * dang) * (dr * ir)
                pts.append(p)
        v0 = np.array(pts).T.copy()
        ov, ob, ost, oie, oit, ot = oracle_track_timed(lat, v0, 0, len(lat), turns, absolute_time=True)
        assert np.array_equal(surv[0, d].reshape(-1), np.where(ost == L.ALIVE, turns, oit))
    assert np.any(surv < turns) and np.any(surv == turns)
