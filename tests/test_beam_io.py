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
