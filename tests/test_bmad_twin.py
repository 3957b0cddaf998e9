"""Bmad lattice files (bgt.bmad_twin): the tracker's lattices written as
Bmad lattice files read back to the same elements, bit for bit in every
attribute and in the tables the tracker compiles from them, and a lattice
in the reference's own element-definition style (inheritance, flag
attributes, expressions) read to the elements the oracle's golden tests
build by hand."""
from __future__ import annotations

import math

import numpy as np
import pytest

from bgt import _lib, bmad_twin, rings
from bgt import lattice as L

from helpers import oracle_track_elements, random_particles, rare_zoo_lattice, zoo_lattice


def _same(a: L.Element, b: L.Element):
    assert a.key == b.key
    for n in L._VALUE_NAMES:
        assert a.v(n) == b.v(n), (a.name, n, a.v(n), b.v(n))
    for f in ("num_steps", "is_on", "fringe_type", "fringe_at", "aperture_type", "aperture_at",
              "offset_moves_aperture", "exact_multipoles", "scale_multipoles", "coupler_at", "has_misalign"):
        assert getattr(a, f) == getattr(b, f), (a.name, f)
    for f in ("a_pole", "b_pole", "ksl_pole", "a_pole_elec", "b_pole_elec"):
        assert {k: v for k, v in getattr(a, f).items() if v} == {k: v for k, v in getattr(b, f).items() if v}


@pytest.mark.parametrize("make", [lambda: rings.fodo_ring(apertures=True), zoo_lattice, rare_zoo_lattice,
                                  lambda: rings.error_variants(1, seed=5)[0]])
def test_write_read_round_trip(make, tmp_path):
    lat = make()
    f = tmp_path / "twin.bmad"
    bmad_twin.write_lattice(lat, str(f))
    back = bmad_twin.read_lattice(str(f))
    assert len(back.elements) == len(lat.elements)
    assert back.p0c == lat.p0c and back.species.charge == lat.species.charge
    for a, b in zip(lat.elements, back.elements):
        _same(a, b)
        assert bytes(_lib.to_bgt_element(a))[8:] == bytes(_lib.to_bgt_element(b))[8:]  # all but key/ix_ele


def test_round_trip_tracks_identically(tmp_path):
    lat = rare_zoo_lattice()
    f = tmp_path / "rz.bmad"
    bmad_twin.write_lattice(lat, str(f), geometry="open")
    back = bmad_twin.read_lattice(str(f))
    v0 = random_particles(256, seed=3)
    a = oracle_track_elements(lat, v0, 0, len(lat), 2, variant="cr")
    b = oracle_track_elements(back, v0, 0, len(back), 2, variant="cr")
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


LATTICE_TEXT = """
! elements written in the style of the reference's element tests
parameter[geometry] = open
parameter[e_tot] = 1e6          ! a positron (Bmad's default species)
k = 0.6
q0: quadrupole, a0 = 0.01, a1 = 0.1, vkick = -0.0001, b0_elec = -2e3, a1_elec = 2e4
quad: q0, l = k, k1 = 1, tilt, num_steps = 10, x_offset = 0.05, y_pitch = 0.001
sext: sextupole, l = 0.6, k2 = 1, tilt, num_steps = 10,
                 x_offset = 0.05, y_pitch = 0.001
mult: multipole, k1l = 1, t1, k3l = 4.5, t3 = 0.31*pi, x_offset = 0.05
coll: ecollimator, l = 4.5, x_limit = 0.2, y_limit = 0.1, num_steps = 10
rb: rbend, l = 0.6, g = 0.01, e1 = 0.1, fint
rf: rfcavity, l = 4.5, rf_frequency = 500e6, voltage = 1e5, phi0 = 0.1, coupler_strength = 0.1, &
    coupler_at = both_ends, cavity_type = traveling_wave
quad[x_offset] = 0.04
cell: line = (quad, sext)
all: line = (cell, mult, coll, rb, rf)
use, all
"""


def test_reads_the_reference_style():
    lat = bmad_twin.read_lattice(LATTICE_TEXT, text=True)
    names = [e.name for e in lat.elements]
    assert names == ["QUAD", "SEXT", "MULT", "COLL", "RB", "RF"]
    assert lat.species.name == "positron" and lat.e_tot == 1e6
    q, s, m, c, b, rf = lat.elements
    assert q.key == "quadrupole" and q.v("l") == 0.6 and q.v("tilt") == math.pi / 4
    assert q.v("x_offset") == 0.04 and q.a_pole == {0: 0.01, 1: 0.1} and q.b_pole_elec == {0: -2e3}
    assert s.v("tilt") == math.pi / 6 and s.user_num_steps == 10
    assert m.a_pole == {1: 1.0, 3: 4.5} and m.b_pole == {1: math.pi / 4, 3: 0.31 * math.pi}
    assert c.v("x1_limit") == c.v("x2_limit") == 0.2 and c.aperture_type == "elliptical"
    assert b.key == "sbend" and b.v("fint") == 0.5 and b.v("l") > 0.6 and b.v("e1") > 0.1
    assert rf.coupler_at == "both_ends" and rf.v("coupler_strength") == 0.1
    # the quadrupole is the golden rows' QUADRUPOLE1 element, with x_offset 0.04
    assert q.v("k1") == 1 and q.v("y_pitch") == 0.001


def test_ltt_init_names_the_files(tmp_path):
    f = tmp_path / "ltt.init"
    bmad_twin.write_ltt_init(str(f), "ring.bmad", "beam.dat", 1000)
    t = f.read_text()
    assert t.startswith("&params") and t.rstrip().endswith("/")
    for s in ("ltt%lat_file = 'ring.bmad'", "beam_init%position_file = 'beam.dat'", "ltt%n_turns = 1000",
              "ltt%tracking_method = 'BMAD'", "ltt%simulation_mode = 'BEAM'"):
        assert s in t


def test_write_twin_files(tmp_path):
    from bgt import beam_io

    lat = rings.fodo_ring(apertures=True)
    v0 = random_particles(50, seed=4)
    files = bmad_twin.write_twin(lat, v0, str(tmp_path), 100)
    back = bmad_twin.read_lattice(files["lattice"])
    assert len(back.elements) == len(lat.elements)
    beam = beam_io.read_ascii_beam(files["beam"])
    assert np.allclose(beam[0].vec6, v0, rtol=1e-15, atol=0)
    assert "ring.bmad" in open(files["init"]).read()


def test_bad_input_is_reported():
    with pytest.raises(ValueError, match="unknown element type"):
        bmad_twin.read_lattice("parameter[e_tot] = 1e9\nx: wiggler, l = 1\nl1: line = (x)\nuse, l1\n", text=True)
    with pytest.raises(ValueError, match="not defined"):
        bmad_twin.read_lattice("parameter[e_tot] = 1e9\nl1: line = (x)\nuse, l1\n", text=True)
    with pytest.raises(ValueError, match="no default tilt"):
        bmad_twin.read_lattice("parameter[e_tot] = 1e9\nd: drift, l = 1, tilt\nl1: line = (d)\nuse, l1\n",
                               text=True)
