"""The tracking kernel's element maps, compiled for the host, against the
oracle -- without a GPU.

tests/device_maps_host.cpp builds the per-particle part of bgt_kernel.cuh
(decode, the element bodies, track1_rec and everything they call) with g++
and -ffp-contract=off, the host counterpart of the device build's
--fmad=false, on tables from the same compiler bgt_create runs
(bgt_compile.h).  IEEE division and square root are correctly rounded on
both sides and every transcendental of a particle coordinate goes through
the correctly rounded bgt::cr, so the host build performs the device's
arithmetic bit for bit: these tests hold the device source to the "cr"
oracle on every machine, the GPU parity suite (test_gpu_parity.py) then
shows that the GPU runs it the same way.  A second build with
AddressSanitizer checks that no map reads outside its table.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from bgt import _lib
from bgt import lattice as L
from bgt import rings
from bgt.track import Bunch

from helpers import oracle_track_elements, random_particles, rare_zoo_lattice, zoo_lattice

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "device_maps_host.cpp"
CXXFLAGS = ["-O2", "-ffp-contract=off", "-std=c++17", "-fPIC", "-shared", "-Wno-unknown-pragmas"]


def _build(out: Path, extra=()) -> Path:
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    subprocess.run([gxx, *CXXFLAGS, *extra, "-o", str(out), str(SRC)], check=True, capture_output=True)
    return out


class HostMaps:
    """bgt_create's tables and the kernel's element maps, run on the host."""

    def __init__(self, lattices, so: Path, absolute_time: bool = False):
        self.lats = [lattices] if isinstance(lattices, L.Lattice) else list(lattices)
        self.lib = C.CDLL(str(so))
        f = self.lib.dmh_track
        f.restype = C.c_int
        f.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_int32,
                      C.c_int32, C.c_int32, C.c_char_p, C.c_int32]
        self.lib.dmh_needs_rare.restype = C.c_int
        self.lib.dmh_needs_rare.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]
        self.n_ele = len(self.lats[0].elements)
        self.arr = (_lib.BgtElement * (self.n_ele * len(self.lats)))()
        for v, lat in enumerate(self.lats):
            for i, e in enumerate(lat.elements):
                self.arr[v * self.n_ele + i] = _lib.to_bgt_element(e)
        lat0 = self.lats[0]
        self.sp = _lib.BgtSpecies(lat0.species.mass, lat0.species.charge, 1, 1e3, 1 if absolute_time else 0, 1)

    @property
    def needs_rare(self) -> bool:
        rc = self.lib.dmh_needs_rare(C.addressof(self.arr), self.n_ele, len(self.lats), C.addressof(self.sp))
        assert rc >= 0
        return rc == 1

    def make_bunch(self, v0, with_time: bool = False) -> Bunch:
        return Bunch.from_vec(v0, self.lats[0].p0c, self.lats[0].species.mass, with_time=with_time)

    def track(self, b: Bunch, rec_begin=0, rec_end=None, turn0=0, n_turns=1, variant=None, kernel=0,
              turns=True):
        rec_end = self.n_ele if rec_end is None else rec_end
        var = None if variant is None else np.ascontiguousarray(variant, np.int32)
        err = C.create_string_buffer(512)
        rc = self.lib.dmh_track(C.addressof(self.arr), self.n_ele, len(self.lats), C.addressof(self.sp),
                                None if var is None else var.ctypes.data, b.vec6.ctypes.data, b.beta.ctypes.data,
                                None if b.t is None else b.t.ctypes.data, b.state.ctypes.data,
                                b.ix_ele_lost.ctypes.data,
                                b.ix_turn_lost.ctypes.data if turns else None, b.n, rec_begin, rec_end, turn0,
                                n_turns, kernel, err, 512)
        assert rc == 0, (rc, err.value)
        return b


@pytest.fixture(scope="module")
def so(tmp_path_factory):
    return _build(tmp_path_factory.mktemp("dmh") / "libdmh.so")


def assert_bitwise(b, ov, ob, ost, oie, oit=None, what=""):
    assert np.array_equal(b.state, ost), f"{what}: state"
    assert np.array_equal(b.ix_ele_lost, oie), f"{what}: loss element"
    if oit is not None:
        assert np.array_equal(b.ix_turn_lost, oit), f"{what}: loss turn"
    assert np.array_equal(b.vec6, ov), f"{what}: coordinates differ (max abs {np.max(np.abs(b.vec6 - ov))})"
    assert np.array_equal(b.beta, ob), f"{what}: beta"


@pytest.mark.parametrize("make", [zoo_lattice, rare_zoo_lattice], ids=["zoo", "rare_zoo"])
@pytest.mark.parametrize("kernel", [0, 1], ids=["picked", "rare"])
def test_each_element_track1_bitwise(so, oracle_lib, make, kernel):
    """track1 through every element of both zoos (all element kinds,
    misalignments, bend geometry, electric fields, edge fringe, couplers,
    apertures), in the kernel instance the host picks and in the RARE one."""
    lat = make()
    hm = HostMaps(lat, so)
    assert hm.needs_rare == (make is rare_zoo_lattice)
    v0 = random_particles(512, seed=31)
    for pos, ele in enumerate(lat.elements):
        b = hm.track(hm.make_bunch(v0.copy()), pos, pos + 1, kernel=kernel, turns=False)
        ov, ob, ost, oie, _ = oracle_track_elements(lat, v0, pos, pos + 1, variant="cr")
        assert_bitwise(b, ov, ob, ost, oie, what=ele.name)


@pytest.mark.parametrize("make", [zoo_lattice, rare_zoo_lattice], ids=["zoo", "rare_zoo"])
def test_turns_with_losses(so, oracle_lib, make):
    lat = make()
    hm = HostMaps(lat, so)
    # neither line closes: the orbit grows turn by turn and particles are
    # lost in every one of the four turns
    v0 = random_particles(1024, seed=32, scale=0.25)
    b = hm.track(hm.make_bunch(v0.copy()), n_turns=4)
    ov, ob, ost, oie, oit = oracle_track_elements(lat, v0, 0, len(lat), 4, variant="cr")
    assert len(np.unique(oit[ost != L.ALIVE])) == 4
    assert_bitwise(b, ov, ob, ost, oie, oit, what=f"{lat.name}, 4 turns")


def test_ring_turns_with_apertures_and_start_turn(so, oracle_lib):
    """The 769-element FODO ring with apertures: 40 turns from turn 7,
    losses at quads and the RF; loss turns are absolute."""
    lat = rings.fodo_ring(apertures=True)
    hm = HostMaps(lat, so)
    assert not hm.needs_rare
    v0 = rings.gaussian_beam(rings.BeamSpec(200, 4e-6, 2e-6, 3e-3, 2e-3, seed=77))
    b = hm.track(hm.make_bunch(v0.copy()), turn0=7, n_turns=40)
    ov, ob, ost, oie, oit = oracle_track_elements(lat, v0, 0, len(lat), 40, variant="cr")
    oit = np.where(ost != L.ALIVE, oit + 7, oit)
    assert (ost != L.ALIVE).sum() > 20
    assert_bitwise(b, ov, ob, ost, oie, oit, "ring, 40 turns")


def test_error_variants_batched(so, oracle_lib):
    """Error variants of the ring (misaligned quads and sextupoles with
    multipole errors), particles interleaved over four variants."""
    lats = rings.error_variants(4, seed=5)
    hm = HostMaps(lats, so)
    n = 240
    v0 = random_particles(n, seed=33, scale=0.5)
    var = np.arange(n, dtype=np.int32) % 4
    b = hm.track(hm.make_bunch(v0.copy()), n_turns=3, variant=var)
    for v in range(4):
        m = var == v
        ov, ob, ost, oie, oit = oracle_track_elements(lats[v], v0[:, m], 0, len(lats[v]), 3, variant="cr")
        sub = Bunch(b.vec6[:, m], b.beta[m], b.state[m], b.ix_ele_lost[m], b.ix_turn_lost[m])
        assert_bitwise(sub, ov, ob, ost, oie, oit, f"variant {v}")


def test_lost_input_particles_are_left_alone(so):
    lat = rings.fodo_ring(apertures=True)
    hm = HostMaps(lat, so)
    v0 = random_particles(30, seed=34)
    b = hm.make_bunch(v0.copy())
    b.state[::3] = L.LOST_NEG_X
    b.ix_ele_lost[::3] = 7
    b.ix_turn_lost[::3] = 2
    hm.track(b, turn0=3, n_turns=2)
    assert np.array_equal(b.vec6[:, ::3], v0[:, ::3])
    assert np.all(b.state[::3] == L.LOST_NEG_X) and np.all(b.ix_ele_lost[::3] == 7)
    assert np.all(b.ix_turn_lost[::3] == 2)


_ASAN_CHILD = r"""
import sys
sys.path[:0] = [{root!r} + "/bmad-ecosystem_b200", {root!r} + "/tests", {root!r}]
import numpy as np
from test_device_maps_host import HostMaps
from helpers import random_particles, rare_zoo_lattice, zoo_lattice
from bgt import rings
from pathlib import Path
so = Path({so!r})
for lat in (zoo_lattice(), rare_zoo_lattice()):
    hm = HostMaps(lat, so)
    for kernel in (0, 1):
        v0 = random_particles(64, seed=35, scale=3.0)
        hm.track(hm.make_bunch(v0), n_turns=2, kernel=kernel)
hm = HostMaps(rings.error_variants(2, seed=6), so)
v0 = random_particles(16, seed=36)
hm.track(hm.make_bunch(v0), n_turns=1, variant=np.arange(16, dtype=np.int32) % 2)
print("ASAN-CLEAN")
"""


def test_no_read_outside_the_tables_under_asan(tmp_path):
    """Every element kind of both zoos, each table in a buffer of its own
    size, under AddressSanitizer: a map that read past its record's table
    would abort the child process."""
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    asan = subprocess.run([gxx, "-print-file-name=libasan.so"], capture_output=True, text=True).stdout.strip()
    if not asan or not os.path.isabs(asan) or not os.path.exists(asan):
        pytest.skip("libasan not available")
    so = _build(tmp_path / "libdmh_asan.so", ["-fsanitize=address", "-fno-omit-frame-pointer", "-g", "-O1"])
    env = dict(os.environ, LD_PRELOAD=asan, ASAN_OPTIONS="detect_leaks=0:abort_on_error=0:exitcode=99")
    r = subprocess.run([sys.executable, "-c", _ASAN_CHILD.format(root=str(ROOT), so=str(so))], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "ASAN-CLEAN" in r.stdout, (r.returncode, r.stderr[-3000:])


def test_golden_rows_on_the_host_build(so):
    """Every tracking_method_test row the library supports, through the
    kernel's element maps built for the host: within the row's tolerance of
    the reference's printed value and bit for bit equal to the correctly
    rounded oracle (the GPU golden test, tests/test_gpu_golden.py, asks the
    same of the GPU)."""
    from test_oracle_golden import ELEMENTS, GOLD, START, check_row, make_element

    for name in sorted(ELEMENTS):
        lat = make_element(name)
        hm = HostMaps(lat, so)
        v0 = np.array(START, dtype=np.float64).reshape(6, 1)
        b = hm.track(hm.make_bunch(v0.copy()), n_turns=1)
        assert b.state[0] == L.ALIVE, name
        check_row(name, b.vec6[:, 0], GOLD["tracking_method"][name])
        ov, ob, ost, _, _ = oracle_track_elements(lat, v0.copy(), 0, 1, 1, variant="cr")
        assert np.array_equal(b.vec6, ov) and np.array_equal(b.beta, ob), name


def test_apertures_that_move_with_bends(so, oracle_lib):
    """offset_moves_aperture on bends with tight limits, so that the frame
    decides hundreds of losses: the curved misaligned geometry at both ends
    (the arc shift by a particle-dependent angle), a bare ref_tilt, the
    straight geometry, elliptical and rectangular."""
    ap = {"x1_limit": 0.004, "x2_limit": 0.0045, "y1_limit": 0.002, "y2_limit": 0.0025}
    E = [L.Element("sbend", "BMISAP", {"l": 0.9, "g": 0.015, "e1": 0.02, "x_offset": 4e-4, "y_offset": -3e-4,
                                       "z_offset": 2e-3, "x_pitch": 2e-4, "y_pitch": 1e-4, "ref_tilt": 0.07, **ap},
                   offset_moves_aperture=True, aperture_at="both_ends"),
         L.Element("sbend", "BROLLAP", {"l": 1.2, "g": -0.02, "roll": 3e-3, "x_offset": 2e-4, **ap},
                   offset_moves_aperture=True, aperture_type="elliptical", aperture_at="exit_end"),
         L.Element("sbend", "BTILTAP", {"l": 0.6, "g": 0.01, "ref_tilt": 0.3, **ap}, offset_moves_aperture=True,
                   aperture_type="elliptical", aperture_at="both_ends"),
         L.Element("sbend", "BSTRAP", {"l": 0.5, "k1": 0.05, "x_offset": 5e-4, "y_pitch": 2e-4, **ap},
                   offset_moves_aperture=True, aperture_at="both_ends")]
    lat = L.Lattice(E, L.Species("electron", L.M_ELECTRON, -1), rings.p0c(), rings.E_TOT, "moving_apertures")
    lat.finalize()
    hm = HostMaps(lat, so)
    assert hm.needs_rare
    v0 = random_particles(2000, seed=37)
    for pos, ele in enumerate(lat.elements):
        b = hm.track(hm.make_bunch(v0.copy()), pos, pos + 1, turns=False)
        ov, ob, ost, oie, _ = oracle_track_elements(lat, v0, pos, pos + 1, variant="cr")
        assert (ost != L.ALIVE).sum() > 200, ele.name
        assert_bitwise(b, ov, ob, ost, oie, what=ele.name)


def test_elements_switched_off(so, oracle_lib):
    """Every element of both zoos with is_on = F (track1_bmad.f90:51-60: an
    off bend keeps its edges with g_tot = 0, everything else but thin
    multipoles becomes a drift), through the host build against the oracle."""
    import copy

    v0 = random_particles(512, seed=38)
    for make in (zoo_lattice, rare_zoo_lattice):
        base = make()
        E = []
        for e in base.elements:
            c = copy.deepcopy(e)
            c.is_on = False
            E.append(c)
        lat = L.Lattice(E, base.species, base.p0c, base.e_tot, base.name + "_off")
        lat.finalize()
        hm = HostMaps(lat, so)
        for pos, ele in enumerate(lat.elements):
            b = hm.track(hm.make_bunch(v0.copy()), pos, pos + 1, turns=False)
            ov, ob, ost, oie, _ = oracle_track_elements(lat, v0, pos, pos + 1, variant="cr")
            assert_bitwise(b, ov, ob, ost, oie, what=ele.name + " (off)")


def test_loss_branches_with_extreme_particles(so, oracle_lib):
    """Particles far outside the beam (30x its size) and hand-made ones past
    the momentum limits (|px| >= 1 + pz: lost_pz in drifts and bodies;
    1 + pz < 0: orbit_too_large), through every element of both zoos, with
    coordinates that may end as NaN compared NaN-aware.  Arguments stay in
    the correctly rounded ranges of bgt::cr (beyond them, e.g. cosh of a
    body phase past 2 when 1 + pz -> 0, both builds use the library and are
    not held to each other)."""
    v0 = random_particles(1024, seed=39, scale=30.0)
    v0[1, :40] = np.linspace(-1.6, 1.6, 40)  # |px| past the total momentum
    v0[5, 40:60] = np.linspace(-2.5, -1.05, 20)  # 1 + pz < 0
    seen = set()
    for make in (zoo_lattice, rare_zoo_lattice):
        lat = make()
        hm = HostMaps(lat, so)
        for pos, ele in enumerate(lat.elements):
            b = hm.track(hm.make_bunch(v0.copy()), pos, pos + 1, turns=False)
            ov, ob, ost, oie, _ = oracle_track_elements(lat, v0, pos, pos + 1, variant="cr")
            assert np.array_equal(b.state, ost), ele.name
            assert np.array_equal(b.ix_ele_lost, oie), ele.name
            assert np.array_equal(b.vec6, ov, equal_nan=True), ele.name
            assert np.array_equal(b.beta, ob, equal_nan=True), ele.name
            seen.update(int(s) for s in np.unique(ost))
    assert {L.ALIVE, L.LOST_NEG_X, L.LOST_POS_X, L.LOST_NEG_Y, L.LOST_POS_Y, L.LOST_PZ} <= seen


@pytest.mark.parametrize("make", [zoo_lattice, rare_zoo_lattice], ids=["zoo", "rare_zoo"])
def test_each_element_alone_picks_a_kernel_that_handles_it(so, oracle_lib, make):
    """Each element alone in a line of its own, so that the host picks the
    kernel instance from that one record: a rare feature missing from the
    RARE selection would run on the lean kernel, which skips it, and differ
    from the oracle.  No zoo element needs the RARE instance; all rare-zoo
    elements do but its drift and the misaligned straight (g = 0) bend, which
    the lean kernel handles."""
    base = make()
    v0 = random_particles(256, seed=40)
    lean = []
    for ele in base.elements:
        lat = L.Lattice([ele], base.species, base.p0c, base.e_tot, ele.name)
        hm = HostMaps(lat, so)
        if not hm.needs_rare:
            lean.append(ele.name)
        b = hm.track(hm.make_bunch(v0.copy()), turns=False)
        ov, ob, ost, oie, _ = oracle_track_elements(lat, v0, 0, 1, variant="cr")
        assert_bitwise(b, ov, ob, ost, oie, what=ele.name + " alone")
    if make is rare_zoo_lattice:
        assert lean == ["D", "BSTRAIGHT"]
    else:
        assert lean == [e.name for e in base.elements]


def test_particle_time_and_absolute_rf_on_the_host_build(so):
    """The particle time t (binary128 in software, bgt_qp.cuh) and the RF
    phase from it under absolute time tracking, through the kernel's own
    element maps built for the host: t bit for bit equal to the oracle's
    quad-precision time and the coordinates to its correctly rounded build,
    on every golden element (relative time, and absolute time for the RF
    rows), both zoos with losses, and the ring with apertures over 40 turns
    in absolute time."""
    from helpers import oracle_track_timed
    from test_oracle_golden import ELEMENTS, GOLD, START, make_element

    cases = []
    for name in sorted(ELEMENTS):
        cases.append((make_element(name), np.array(START, dtype=np.float64).reshape(6, 1), 1, False, name))
        if name in GOLD["tracking_method_abs_time"]:
            cases.append((make_element(name), np.array(START, dtype=np.float64).reshape(6, 1), 1, True,
                          name + " abs"))
    cases.append((zoo_lattice(), random_particles(600, seed=41, scale=3.0), 3, False, "zoo"))
    cases.append((rare_zoo_lattice(), random_particles(600, seed=42, scale=0.1), 3, True, "rare zoo abs"))
    cases.append((rings.fodo_ring(apertures=True),
                  rings.gaussian_beam(rings.BeamSpec(400, 4e-6, 2e-6, 3e-3, 2e-3, seed=43)), 40, True, "ring abs"))
    for lat, v0, turns, abs_t, what in cases:
        hm = HostMaps(lat, so, absolute_time=abs_t)
        b = hm.track(hm.make_bunch(v0.copy(), with_time=True), n_turns=turns)
        ov, ob, ost, oie, oit, ot = oracle_track_timed(lat, v0.copy(), 0, len(lat), turns, absolute_time=abs_t)
        assert_bitwise(b, ov, ob, ost, oie, oit, what)
        assert np.array_equal(b.t, ot), what
    assert (ost != L.ALIVE).sum() > 0  # the ring case loses particles
