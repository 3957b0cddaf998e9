"""Bmad ASCII beam files and exact checkpoints (bgt.beam_io), on the CPU."""
from __future__ import annotations

import numpy as np
import pytest

from bgt import beam_io as B
from bgt import lattice as L
from bgt import rings
from bgt.track import Bunch


def _bunch(n=40, seed=1):
    rng = np.random.default_rng(seed)
    v = rings.gaussian_beam(rings.CONFIG0_BEAM, n=n)
    st = np.ones(n, np.int32)
    st[:9] = np.arange(9)  # every state code once
    ixe = np.where(st == 1, -1, rng.integers(1, 700, n)).astype(np.int32)
    beta = L.beta_of(rings.p0c(), v[5], L.M_ELECTRON)
    return Bunch(np.ascontiguousarray(v), beta, st, ixe, np.full(n, -1, np.int32))


def test_ascii_round_trip(tmp_path):
    b = _bunch()
    bb = B.BeamBunch.from_bunch(b, rings.p0c(), species="electron", charge=1e-12)
    f = tmp_path / "beam.dat"
    B.write_ascii_beam(str(f), [bb, bb])
    got = B.read_ascii_beam(str(f))
    assert len(got) == 2
    for g in got:
        assert g.n == b.n and g.species == "electron"
        assert np.allclose(g.vec6, b.vec6, rtol=6e-16, atol=1e-300)
        assert np.array_equal(g.state, b.state)
        assert np.array_equal(g.ix_ele[b.state != 1], b.ix_ele_lost[b.state != 1])
        assert np.all(g.p0c == rings.p0c()) and np.all(g.charge == 1e-12)
    text = f.read_text().splitlines()
    assert text[0] == "# ix_bunch       =     1" and text[4].startswith("# charge         =")
    col = [ln for ln in text if ln.startswith("#!")][0].split()
    assert col == ["#!", "index", "x", "px", "y", "py", "z", "pz", "p0c", "s_position", "time", "spin_x", "spin_y",
                   "spin_z", "state", "ix_ele", "location"]


def test_state_names_follow_the_reference_table(tmp_path):
    b = _bunch()
    bb = B.BeamBunch.from_bunch(b, rings.p0c())
    f = tmp_path / "beam.dat"
    B.write_ascii_beam(str(f), [bb])
    rows = [ln.split() for ln in f.read_text().splitlines() if not ln.startswith("#")]
    # code 7 (lost_z) is written 'Lost_Pz' and code 8 (lost_pz) 'Lost_Z', as
    # the reference's state_name table has them, and read back to the codes
    assert rows[7][-3] == "Lost_Pz" and rows[8][-3] == "Lost_Z" and rows[1][-3] == "Alive"
    assert np.array_equal(B.read_ascii_beam(str(f))[0].state, b.state)


def test_reads_a_file_in_the_reference_layout(tmp_path):
    # header keys tabbed to column 18, a per-particle charge column,
    # Fortran's E-less three-digit exponent, lower-case state names
    txt = """# ix_bunch       =     1
# n_particle     =     2
# n_alive        =     1
# n_dead         =     1
# species         = positron
#!  index                      x                     px                      y                     py                      z                     pz                    p0c                 charge          state
       1  1.000000000000000E-03  0.000000000000000E+00 -2.000000000000000E-04  1.0000000000000000-100  3.000000000000000E-03 -1.000000000000000E-03  4.999999973888e+09  1.000000000000000E-12          alive
       2  2.000000000000000E-02  0.000000000000000E+00  0.000000000000000E+00  0.000000000000000E+00  0.000000000000000E+00  0.000000000000000E+00  4.999999973888e+09  2.000000000000000E-12     Lost_Pos_X
"""
    f = tmp_path / "ref.dat"
    f.write_text(txt)
    (g,) = B.read_ascii_beam(str(f))
    assert g.n == 2 and g.species == "positron"
    assert g.vec6[3, 0] == 1e-100 and g.vec6[2, 0] == -2e-4
    assert list(g.state) == [1, 4] and list(g.charge) == [1e-12, 2e-12]
    tb = g.to_bunch()
    assert np.allclose(tb.beta, L.beta_of(g.p0c, g.vec6[5], L.M_ELECTRON), rtol=0, atol=0)


def test_unknown_column_is_an_error(tmp_path):
    f = tmp_path / "bad.dat"
    f.write_text("#!  x  px  y  py  z  pz  bogus\n 0 0 0 0 0 0 1\n")
    with pytest.raises(ValueError, match="bogus"):
        B.read_ascii_beam(str(f))


def test_checkpoint_is_exact(tmp_path):
    b = _bunch()
    f = tmp_path / "ck.npz"
    B.save_checkpoint(str(f), b, 1234, lattice="fodo64")
    c, turn, meta = B.load_checkpoint(str(f))
    assert turn == 1234 and str(meta["lattice"]) == "fodo64"
    for k in ("vec6", "beta", "state", "ix_ele_lost", "ix_turn_lost"):
        assert np.array_equal(getattr(c, k), getattr(b, k)) and getattr(c, k).dtype == getattr(b, k).dtype


def test_legacy_ascii3_round_trip(tmp_path):
    rng = np.random.default_rng(5)
    n = 40
    vec = rng.standard_normal((6, n)) * 1e-3
    state = np.ones(n, np.int32)
    state[::7] = B.STATE_NAME.index("Lost_Pos_Y")
    b = B.BeamBunch(vec, state, np.full(n, 5e9), np.zeros(n), np.zeros(n), np.full(n, 1e-15),
                          rng.standard_normal((3, n)), np.arange(n, dtype=np.int32), None, "electron",
                          charge_tot=4e-14)
    f = tmp_path / "beam3.dat"
    B.write_ascii3_beam(str(f), [b, b])
    assert f.read_text().startswith("!ASCII::3")
    back = B.read_beam(str(f), p0c=5e9)
    assert len(back) == 2
    for r in back:
        assert r.species == "electron" and r.charge_tot == 4e-14
        assert np.allclose(r.vec6, vec, rtol=1e-10, atol=0)
        assert np.array_equal(r.state, state) and np.array_equal(r.ix_ele, b.ix_ele)
        assert np.allclose(r.spin, b.spin, rtol=1e-10) and np.all(r.p0c == 5e9)


def test_legacy_ascii3_short_lines_and_extra_particles(tmp_path):
    f = tmp_path / "short.dat"
    f.write_text("""!ASCII::3
 5   ! ix_ele
 1   ! n_bunch
 2   ! n_particle
 BEGIN_BUNCH
   positron
 1e-12  ! charge_tot
 0.0  ! z_center
 0.0  ! t_center
 1e-3 2e-4 -1e-3 0 0.01 1e-3
 2e-3 0 0 0 0 0  1.0E-15  6
 9 9 9 9 9 9
 END_BUNCH
""")
    (b,) = B.read_beam(str(f), p0c=1e9)
    assert b.n == 2 and b.species == "positron"
    assert np.array_equal(b.vec6[:, 0], [1e-3, 2e-4, -1e-3, 0, 0.01, 1e-3])
    assert b.state[0] == 1 and b.state[1] == 6 and b.charge[1] == 1e-15
    assert np.all(b.ix_ele == 5)


def test_read_beam_tells_the_formats_apart(tmp_path):
    bunch = Bunch.from_vec(np.full((6, 3), 1e-3), 1e9, B.SPECIES_MASS["electron"])
    f = tmp_path / "new.dat"
    B.write_ascii_beam(str(f), [B.BeamBunch.from_bunch(bunch, 1e9)])
    assert B.read_beam(str(f))[0].n == 3
    g = tmp_path / "bin.dat"
    g.write_text("!BIN::3\n")  # tagged binary, but not framed as records
    with pytest.raises(ValueError, match="framing|ends"):
        B.read_beam(str(g))


def _bin3_bunch(n=30, seed=6, species="positron"):
    rng = np.random.default_rng(seed)
    state = np.ones(n, np.int32)
    state[::5] = B.STATE_NAME.index("Lost_Neg_X")
    return B.BeamBunch(rng.standard_normal((6, n)) * 1e-3, state, np.full(n, 5e9), np.zeros(n), np.zeros(n),
                       rng.uniform(1e-16, 2e-16, n), rng.standard_normal((3, n)), np.full(n, 12, np.int32), None,
                       species, charge_tot=3e-14)


def test_bin3_round_trip_is_exact_and_detected(tmp_path):
    a, b = _bin3_bunch(), _bin3_bunch(seed=7, species="electron")
    f = tmp_path / "beam.bin"
    B.write_bin3_beam(str(f), [a, b])
    back = B.read_beam(str(f), p0c=5e9)
    assert [r.species for r in back] == ["positron", "electron"]
    for r, w in zip(back, (a, b)):
        assert np.array_equal(r.vec6, w.vec6) and np.array_equal(r.spin, w.spin)
        assert np.array_equal(r.charge, w.charge) and np.array_equal(r.state, w.state)
        assert r.charge_tot == 3e-14 and r.location == "Downstream_End" and np.all(r.ix_ele == 12)


def test_bin3_record_layout(tmp_path):
    """gfortran unformatted sequential records, each framed by its 4-byte
    length: the 7-byte tag, 3 integers, per bunch an integer species code,
    three reals and an integer, per particle 6 + 1 reals, an integer, 3
    reals and two integers (beam_file_io.f90:483-495, 652-667)."""
    import struct

    f = tmp_path / "beam.bin"
    B.write_bin3_beam(str(f), [_bin3_bunch(n=2)])
    data = f.read_bytes()
    sizes, pos = [], 0
    while pos < len(data):
        (n,) = struct.unpack_from("<i", data, pos)
        assert struct.unpack_from("<i", data, pos + 4 + n)[0] == n
        sizes.append(n)
        pos += 8 + n
    assert sizes == [7, 12, 32, 92, 92]
    assert data[4:11] == b"!BIN::3"
    assert struct.unpack_from("<iii", data, 19) == (12, 1, 2)
    assert struct.unpack_from("<i", data, 39)[0] == 1  # positron$ = +1


def test_bin3_errors_and_old_binary(tmp_path):
    f = tmp_path / "beam.bin"
    B.write_bin3_beam(str(f), [_bin3_bunch(n=4)])
    data = f.read_bytes()
    (tmp_path / "cut.bin").write_bytes(data[:-10])
    with pytest.raises(ValueError, match="framing|ends"):
        B.read_beam(str(tmp_path / "cut.bin"))
    (tmp_path / "old.bin").write_bytes(b"\x07\x00\x00\x00!BIN::2\x07\x00\x00\x00")
    with pytest.raises(ValueError, match="old style binary"):
        B.read_beam(str(tmp_path / "old.bin"))


def test_normalized_charge_follows_read_beam_file():
    b = _bin3_bunch(n=4)
    q = b.normalized_charge()
    assert np.isclose(q.sum(), 3e-14, rtol=1e-15) and np.allclose(q / b.charge, q[0] / b.charge[0])
    b.charge[:] = 0
    assert np.all(b.normalized_charge() == 3e-14 / 4)
    b.charge_tot = 0.0
    assert np.all(b.normalized_charge() == 0)
