"""Beam files and checkpoints for the tracker's particle arrays.

* Bmad's ASCII beam format, written as ``write_ascii_beam_file`` and read as
  ``read_beam_ascii`` do (bmad/multiparticle/beam_file_io.f90:123-350 and
  :834-1275): per bunch a header of ``# key = value`` lines, a ``#!`` column
  line and one row per particle (``es23.15`` reals).  Columns that hold the
  same value for every particle (charge, species, ix_branch, direction,
  time_dir) move to the header, all-zero field / phase / dt_ref columns are
  dropped, spin is always written (:185-195).  Particle states are written and
  read with the reference's ``state_name`` table (bmad_struct.f90:535-536),
  whose entries 7 and 8 read 'Lost_Pz' and 'Lost_Z' while the codes are
  lost_z = 7 and lost_pz = 8: files written by Bmad round-trip through this
  module unchanged.  ``es23.15`` keeps 16 significant digits, so an ASCII
  round trip moves coordinates by up to ~5e-16 relative.
* The legacy ``!ASCII::3`` format (``write_ascii3_beam`` /
  ``read_ascii3_beam``), its binary twin ``!BIN::3`` (``write_bin3_beam`` /
  ``read_bin3_beam``: gfortran unformatted sequential records, as
  ``read_beam_file`` reads them, beam_file_io.f90:483-495, 652-667), and
  ``read_beam``, which tells the formats apart as ``read_beam_file`` does.
  Per-particle charges are returned as stored, with the bunch's charge_tot;
  ``BeamBunch.normalized_charge`` applies read_beam_file's rescaling
  (:685-693).
* Checkpoints (``save_checkpoint`` / ``load_checkpoint``): the exact FP64 /
  int32 arrays and the next turn index in one ``.npz`` file, so that tracking
  resumed from a checkpoint (``turn0`` = the saved turn) is bit-identical to
  an uninterrupted run -- the role of long_term_tracking's restart from a
  saved beam (``ltt%ix_turn_start``, bsim/modules/lt_tracking_mod.f90).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass
from typing import Dict, List, Optional

import numpy as np

from .track import Bunch

# bmad_struct.f90:535-536 (zero based); note the order of entries 7 and 8
STATE_NAME = ["Pre_Born", "Alive", "Lost", "Lost_Neg_X", "Lost_Pos_X", "Lost_Neg_Y", "Lost_Pos_Y", "Lost_Pz",
              "Lost_Z"]
# bmad_struct.f90:398-399
LOCATION_NAME = ["GARBAGE!", "Upstream_End", "Downstream_End", "Inside"]
# integer species codes (sim_utils/interfaces/particle_species_mod.f90:64-68)
SPECIES_ID = {"proton": 2, "positron": 1, "electron": -1, "antiproton": -2}
# species names (physical_constants / particle_species_mod), the ones this tracker handles
SPECIES_MASS = {"electron": 0.51099895069e6, "positron": 0.51099895069e6, "proton": 938.27208816e6,
                "antiproton": 938.27208816e6}


@dataclass
class BeamBunch:
    """One bunch of a beam file: coordinates and per-particle bookkeeping."""
    vec6: np.ndarray  # (6, n)
    state: np.ndarray  # int32 (n,)
    p0c: np.ndarray  # (n,)
    s: np.ndarray
    t: np.ndarray
    charge: np.ndarray
    spin: np.ndarray  # (3, n)
    ix_ele: np.ndarray  # int32
    beta: Optional[np.ndarray] = None
    species: str = "electron"
    location: str = "Downstream_End"
    ix_branch: int = 0
    direction: int = 1
    time_dir: int = 1
    charge_tot: Optional[float] = None

    @property
    def n(self) -> int:
        return self.vec6.shape[1]

    @classmethod
    def from_bunch(cls, b: Bunch, p0c: float, species: str = "electron", s: float = 0.0, t: float = 0.0,
                   charge: float = 0.0) -> "BeamBunch":
        n = b.n
        return cls(np.array(b.vec6, dtype=np.float64), np.array(b.state, np.int32), np.full(n, p0c),
                   np.full(n, s), np.full(n, t), np.full(n, charge), np.zeros((3, n)),
                   np.array(b.ix_ele_lost, np.int32), np.array(b.beta), species)

    def normalized_charge(self) -> np.ndarray:
        """Per-particle charges as read_beam_file leaves them
        (beam_file_io.f90:685-693): scaled so that they sum to charge_tot,
        or charge_tot / n each when the file gives none."""
        q = np.asarray(self.charge, dtype=np.float64)
        tot = self.charge_tot if self.charge_tot is not None else 0.0
        s = 0.0
        for v in q:  # Fortran sum order
            s = s + v
        if tot == 0:
            return q.copy()
        if s == 0:
            return np.full(q.shape, tot / self.n)
        return q * tot / s

    def to_bunch(self) -> Bunch:
        """Tracker arrays; beta from the file or, as the reader's
        bunch_finalizer does, from (1 + pz) p0c and the species mass."""
        beta = self.beta
        if beta is None:
            pc = (1 + self.vec6[5]) * self.p0c
            m = SPECIES_MASS[self.species.lower()]
            beta = pc / np.sqrt(pc * pc + m * m)
        n = self.n
        ixe = np.where(self.state == 1, -1, self.ix_ele).astype(np.int32)
        return Bunch(np.ascontiguousarray(self.vec6, dtype=np.float64), np.ascontiguousarray(beta, np.float64),
                     np.ascontiguousarray(self.state, np.int32), ixe, np.full(n, -1, np.int32))


def _key(who: str) -> str:
    return ("# " + who).ljust(17)


def _es(v: float) -> str:
    """Fortran es23.15."""
    return f"{v:23.15E}"


def write_ascii_beam(path: str, bunches: List[BeamBunch], new_file: bool = True, alive_only: bool = False):
    cols = ["index", "vec", "p0c", "s_position", "time", "charge", "spin", "state", "ix_ele", "ix_branch",
            "location", "species", "direction", "time_dir"]
    # constant columns go to the header (the reference's remove_col rules)
    const = {"charge": all(np.all(b.charge == b.charge[0]) for b in bunches if b.n),
             "species": True, "ix_branch": True, "direction": True, "time_dir": True}
    for k, c in const.items():
        if c:
            cols.remove(k)
    with open(path, "w" if new_file else "a") as f:
        for ib, b in enumerate(bunches, 1):
            keep = np.ones(b.n, bool) if not alive_only else (b.state == 1) | (b.state == 0)
            n_alive = int(np.sum((b.state == 1) | (b.state == 0)))
            f.write(f"# ix_bunch       ={ib:6d}\n")
            f.write(f"# n_particle     ={b.n:6d}\n")
            f.write(f"# n_alive        ={n_alive:6d}\n")
            f.write(f"# n_dead         ={b.n - n_alive:6d}\n")
            # headwrite_re / _int / _str: the key tabbed to column 18
            if "charge" not in cols:
                f.write(_key("charge") + f"={(b.charge[0] if b.n else 0.0):24.16E}\n")
            f.write(_key("ix_branch") + f"= {b.ix_branch}\n")
            f.write(_key("direction") + f"= {b.direction}\n")
            f.write(_key("time_dir") + f"= {b.time_dir}\n")
            f.write(_key("species") + f"= {b.species}\n")
            head = ""
            for c in cols:
                if c in ("index", "ix_ele"):
                    head += f"{c:>8}"
                elif c == "vec":
                    head += "".join(f"{x:>23}" for x in ("x", "px", "y", "py", "z", "pz"))
                elif c in ("p0c", "s_position", "time", "charge"):
                    head += f"{c:>23}"
                elif c == "spin":
                    head += "".join(f"{x:>23}" for x in ("spin_x", "spin_y", "spin_z"))
                elif c == "state":
                    head += f"{c:>14}"
                elif c == "location":
                    head += f"{c:>16}"
            f.write("#!" + head[2:] + "\n")
            for ip in range(b.n):
                if not keep[ip]:
                    continue
                row = ""
                for c in cols:
                    if c == "index":
                        row += f"{ip + 1:8d}"
                    elif c == "vec":
                        row += "".join(_es(v) for v in b.vec6[:, ip])
                    elif c == "p0c":
                        row += _es(b.p0c[ip])
                    elif c == "s_position":
                        row += _es(b.s[ip])
                    elif c == "time":
                        row += _es(b.t[ip])
                    elif c == "charge":
                        row += _es(b.charge[ip])
                    elif c == "spin":
                        row += "".join(_es(v) for v in b.spin[:, ip])
                    elif c == "state":
                        row += f"{STATE_NAME[int(b.state[ip])]:>14}"
                    elif c == "ix_ele":
                        row += f"{int(b.ix_ele[ip]):8d}"
                    elif c == "location":
                        row += f"{b.location:>16}"
                f.write(row.rstrip() + "\n")


def _float(tok: str) -> float:
    t = tok.strip().replace("D", "E").replace("d", "e")
    try:
        return float(t)
    except ValueError:
        # Fortran drops the 'E' for three-digit exponents: 1.0-100
        for i in range(len(t) - 1, 0, -1):
            if t[i] in "+-" and t[i - 1] not in "eE":
                return float(t[:i] + "E" + t[i:])
        raise


def _match(name: str, table: List[str], what: str) -> int:
    for i, s in enumerate(table):
        if s.lower() == name.strip().strip("'\"").lower():
            return i
    raise ValueError(f"{what} name not recognised: {name!r}")


def read_ascii_beam(path: str) -> List[BeamBunch]:
    """Every bunch of an ASCII beam file."""
    lines = open(path).read().splitlines()
    out: List[BeamBunch] = []
    i = 0
    while i < len(lines):
        hdr: Dict[str, str] = {}
        cols: Optional[List[str]] = None
        while i < len(lines):
            ln = lines[i]
            i += 1
            if ln.strip() == "":
                continue
            if ln.startswith("#!"):
                cols = ln[2:].split()
                break
            if not ln.startswith("#"):
                raise ValueError(f"header line does not start with '#': {ln[:20]!r}")
            if "=" in ln:
                k, v = ln[1:].split("=", 1)
                hdr[k.strip().lower()] = v.strip()
        if cols is None:
            break
        rows = []
        while i < len(lines):
            ln = lines[i]
            if ln.strip() == "":
                i += 1
                continue
            if ln.startswith("#"):
                break
            rows.append(ln.split())
            i += 1
        n = len(rows)
        species = hdr.get("species", "positron").strip("'\"")
        p0 = {"p0c": _float(hdr["p0c"]) if "p0c" in hdr else 0.0,
              "s": _float(hdr.get("s", hdr.get("s_position", "0"))), "t": _float(hdr.get("t", hdr.get("time", "0"))),
              "charge": _float(hdr.get("charge", "0"))}
        b = BeamBunch(np.zeros((6, n)), np.full(n, _match(hdr["state"], STATE_NAME, "state") if "state" in hdr
                                                 else 1, np.int32),
                      np.full(n, p0["p0c"]), np.full(n, p0["s"]), np.full(n, p0["t"]), np.full(n, p0["charge"]),
                      np.zeros((3, n)), np.zeros(n, np.int32), None, species,
                      hdr.get("location", "Downstream_End"), int(_float(hdr.get("ix_branch", "0"))),
                      int(_float(hdr.get("direction", "1"))), int(_float(hdr.get("time_dir", "1"))),
                      _float(hdr["charge_tot"]) if "charge_tot" in hdr else None)
        if "beta" in hdr:
            b.beta = np.full(n, _float(hdr["beta"]))
        vec_idx = {"x": 0, "px": 1, "y": 2, "py": 3, "z": 4, "pz": 5}
        spin_idx = {"spin_x": 0, "spin_y": 1, "spin_z": 2}
        for ip, r in enumerate(rows):
            if len(r) < len(cols):
                raise ValueError(f"row {ip + 1} of a bunch has {len(r)} entries for {len(cols)} columns")
            for c, tok in zip(cols, r):
                cl = c.lower()
                if cl in vec_idx:
                    b.vec6[vec_idx[cl], ip] = _float(tok)
                elif cl in spin_idx:
                    b.spin[spin_idx[cl], ip] = _float(tok)
                elif cl == "p0c":
                    b.p0c[ip] = _float(tok)
                elif cl in ("s", "s_position"):
                    b.s[ip] = _float(tok)
                elif cl in ("t", "time"):
                    b.t[ip] = _float(tok)
                elif cl == "charge":
                    b.charge[ip] = _float(tok)
                elif cl == "beta":
                    if b.beta is None:
                        b.beta = np.zeros(n)
                    b.beta[ip] = _float(tok)
                elif cl == "state":
                    b.state[ip] = _match(tok, STATE_NAME, "state")
                elif cl == "ix_ele":
                    b.ix_ele[ip] = int(tok)
                elif cl == "location":
                    b.location = LOCATION_NAME[_match(tok, LOCATION_NAME, "location")]
                elif cl == "species":
                    b.species = tok
                elif cl == "index":
                    int(tok)  # must be an integer; value unused
                elif cl in ("ix_branch", "direction", "time_dir", "ix_user"):
                    int(tok)
                elif cl in ("field_x", "field_y", "phase_x", "phase_y", "dt_ref", "r", "e_potential"):
                    _float(tok)
                else:
                    raise ValueError(f"column name not recognised: {c}")
        out.append(b)
    return out


# ---------------------------------------------------------------------------
# The legacy '!ASCII::3' format: write_beam_file with old_ascii$ and the
# ASCII::3 branch of read_beam_file (bmad/multiparticle/beam_file_io.f90:76-106,
# 446-640).  Header: ix_ele, n_bunch, n_particle; per bunch BEGIN_BUNCH, the
# species, charge_tot, z_center, t_center, one line per particle
# (6es19.10 coordinates, es14.5 charge, i6 state, 3es19.10 spin, i6 ix_ele,
# i3 location) and END_BUNCH.  Reading, a particle line needs the six
# coordinates and may stop after any later field; lines beyond n_particle
# are skipped.  p0c is not part of the format: the caller gives it.

def write_ascii3_beam(path: str, bunches: List[BeamBunch], new_file: bool = True) -> None:
    with open(path, "w" if new_file else "a") as f:
        if new_file:
            f.write("!ASCII::3\n")
        first = bunches[0] if bunches else None
        ix_ele = int(first.ix_ele[0]) if first is not None and first.n else 0
        f.write(f"  {ix_ele}  ! ix_ele\n  {len(bunches)}  ! n_bunch\n  {first.n if first else 0}  ! n_particle\n")
        for b in bunches:
            loc = LOCATION_NAME.index(b.location) if b.location in LOCATION_NAME else 2
            charge_tot = b.charge_tot if b.charge_tot is not None else float(np.sum(b.charge))
            f.write(" BEGIN_BUNCH\n")
            f.write(f"   {b.species}\n")
            f.write(f"  {charge_tot!r}  ! charge_tot\n  0.0  ! z_center\n  0.0  ! t_center\n")
            for j in range(b.n):
                f.write("".join(f"{v:19.10E}" for v in b.vec6[:, j]) + f"{b.charge[j]:14.5E}{int(b.state[j]):6d}" +
                        "".join(f"{v:19.10E}" for v in b.spin[:, j]) + f"{int(b.ix_ele[j]):6d}{loc:3d}\n")
            f.write(" END_BUNCH\n")


def read_ascii3_beam(path: str, p0c: float = 0.0) -> List[BeamBunch]:
    words = []
    for ln in open(path).read().splitlines():
        if ln.strip().upper().startswith("!ASCII::3"):
            continue
        body = ln.split("!", 1)[0].strip()
        if body:
            words.append(body)
    it = iter(words)

    def nxt(what):
        try:
            return next(it)
        except StopIteration:
            raise ValueError(f"beam file ends before the {what}") from None

    ix_ele = int(_float(nxt("ix_ele")))
    n_bunch = int(_float(nxt("n_bunch")))
    n_particle = int(_float(nxt("n_particle")))
    out = []
    for _ in range(n_bunch):
        if "BEGIN_BUNCH" not in nxt("BEGIN_BUNCH marker").upper():
            raise ValueError('no "BEGIN_BUNCH" marker found')
        species = nxt("species").split()[0]
        try:
            _float(species)
            numeric = True
        except ValueError:
            numeric = False
        if numeric:
            raise ValueError("old style format does not include the bunch species")
        charge_tot = _float(nxt("charge_tot"))
        nxt("z_center")
        nxt("t_center")
        vec = np.zeros((6, n_particle))
        charge = np.zeros(n_particle)
        state = np.ones(n_particle, np.int32)
        spin = np.zeros((3, n_particle))
        ixe = np.full(n_particle, ix_ele, np.int32)
        loc = 2
        j = 0
        while True:
            ln = nxt("END_BUNCH marker")
            if "END_BUNCH" in ln.upper():
                break
            if j >= n_particle:
                j += 1
                continue
            tok = ln.replace("(", " ").replace(")", " ").replace(",", " ").split()
            if len(tok) < 6:
                raise ValueError(f"particle line with fewer than 6 coordinates: {ln!r}")
            vec[:, j] = [_float(t) for t in tok[:6]]
            if len(tok) > 6:
                charge[j] = _float(tok[6])
            if len(tok) > 7:
                state[j] = int(tok[7])
            if len(tok) > 10:
                spin[:, j] = [_float(t) for t in tok[8:11]]
            if len(tok) > 11:
                ixe[j] = int(tok[11])
            if len(tok) > 12:
                loc = int(tok[12])
            j += 1
        if j < n_particle:
            raise ValueError(f"bunch has {j} particle lines for n_particle = {n_particle}")
        out.append(BeamBunch(vec, state, np.full(n_particle, p0c), np.zeros(n_particle), np.zeros(n_particle),
                             charge, spin, ixe, None, species.lower(), LOCATION_NAME[loc], charge_tot=charge_tot))
    return out


_BIN3_BUNCH = struct.Struct("<idddi")  # species, charge_tot, z_center, t_center, n_particle_lines
_BIN3_PART = struct.Struct("<6ddi3dii")  # vec, charge, state, spin, ix_ele, location


def _fortran_record(payload: bytes) -> bytes:
    n = struct.pack("<i", len(payload))
    return n + payload + n


def write_bin3_beam(path: str, bunches: List[BeamBunch]) -> None:
    """The ``!BIN::3`` layout read_beam_file reads (beam_file_io.f90:483-495,
    652-667): gfortran unformatted sequential records, each framed by its
    4-byte length -- the tag, (ix_ele, n_bunch, n_particle), then per bunch
    (species, charge_tot, z_center, t_center, n) and one record per particle
    (vec, charge, state, spin, ix_ele, location)."""
    first = bunches[0] if bunches else None
    ix_ele = int(first.ix_ele[0]) if first is not None and first.n else 0
    with open(path, "wb") as f:
        f.write(_fortran_record(b"!BIN::3"))
        f.write(_fortran_record(struct.pack("<iii", ix_ele, len(bunches), first.n if first else 0)))
        for b in bunches:
            loc = LOCATION_NAME.index(b.location) if b.location in LOCATION_NAME else 2
            charge_tot = b.charge_tot if b.charge_tot is not None else float(np.sum(b.charge))
            f.write(_fortran_record(_BIN3_BUNCH.pack(SPECIES_ID[b.species.lower()], charge_tot, 0.0, 0.0, b.n)))
            for j in range(b.n):
                f.write(_fortran_record(_BIN3_PART.pack(*b.vec6[:, j], b.charge[j], int(b.state[j]), *b.spin[:, j],
                                                        int(b.ix_ele[j]), loc)))


def read_bin3_beam(path: str, p0c: float = 0.0) -> List[BeamBunch]:
    """A ``!BIN::3`` beam file (see write_bin3_beam); p0c is not stored in the
    format and is taken from the caller."""
    data = open(path, "rb").read()
    pos = 0

    def record(what):
        nonlocal pos
        if pos + 4 > len(data):
            raise ValueError(f"beam file ends before the {what}")
        (n,) = struct.unpack_from("<i", data, pos)
        if n < 0 or pos + 8 + n > len(data) or struct.unpack_from("<i", data, pos + 4 + n)[0] != n:
            raise ValueError(f"bad record framing at the {what}")
        out = data[pos + 4:pos + 4 + n]
        pos += 8 + n
        return out

    if record("tag")[:7] != b"!BIN::3":
        raise ValueError("not a !BIN::3 beam file")
    ix_ele, n_bunch, n_particle = struct.unpack_from("<iii", record("header"))
    id_to_name = {v: k for k, v in SPECIES_ID.items()}
    out = []
    for _ in range(n_bunch):
        species, charge_tot, _z, _t, n_lines = _BIN3_BUNCH.unpack_from(record("bunch parameters"))
        if species not in id_to_name:
            raise ValueError(f"species code {species} is not handled")
        vec = np.zeros((6, n_particle))
        charge = np.zeros(n_particle)
        state = np.ones(n_particle, np.int32)
        spin = np.zeros((3, n_particle))
        ixe = np.full(n_particle, ix_ele, np.int32)
        loc = 2
        j = 0
        for j in range(1, n_lines + 1):
            v = _BIN3_PART.unpack_from(record("particle coordinates"))
            vec[:, j - 1] = v[0:6]
            charge[j - 1] = v[6]
            state[j - 1] = v[7]
            spin[:, j - 1] = v[8:11]
            loc = v[12]  # the particle's ix_ele is read into a scratch variable (:658)
            if j == n_particle:
                break
        if j < n_particle:
            raise ValueError(f"bunch has {j} particle records for n_particle = {n_particle}")
        out.append(BeamBunch(vec, state, np.full(n_particle, p0c), np.zeros(n_particle), np.zeros(n_particle),
                             charge, spin, ixe, None, id_to_name[species], LOCATION_NAME[loc],
                             charge_tot=charge_tot))
    return out


def read_beam(path: str, p0c: float = 0.0) -> List[BeamBunch]:
    """A beam file in any of the formats, told apart as read_beam_file does
    (beam_file_io.f90:455-476) from its first 80 characters: '!BIN::3' is
    the binary legacy format ('!BINARY' / '!BIN::2', older still, are
    refused), '!ASCII::3' (or a first non-blank line that is not a '#'
    header) the ASCII legacy format, '#' starts the current one.  p0c is
    used by the legacy formats only."""
    head = open(path, "rb").read(80)
    if b"!BINARY" in head or b"!BIN::2" in head:
        raise ValueError("old style binary beam files are not supported")
    if b"!BIN::3" in head:
        return read_bin3_beam(path, p0c)
    with open(path) as f:
        first = ""
        for ln in f:
            if ln.strip():
                first = ln
                break
    if first.startswith("#"):
        return read_ascii_beam(path)
    return read_ascii3_beam(path, p0c)


def save_checkpoint(path: str, bunch: Bunch, next_turn: int, **meta):
    """Exact tracker state and the index of the next turn to track."""
    np.savez(path, vec6=bunch.vec6, beta=bunch.beta, state=bunch.state, ix_ele_lost=bunch.ix_ele_lost,
             ix_turn_lost=bunch.ix_turn_lost, next_turn=np.int64(next_turn),
             **{k: np.asarray(v) for k, v in meta.items()})


def load_checkpoint(path: str):
    """(Bunch, next_turn, meta) from save_checkpoint."""
    z = np.load(path)
    b = Bunch(np.ascontiguousarray(z["vec6"]), np.ascontiguousarray(z["beta"]), np.ascontiguousarray(z["state"]),
              np.ascontiguousarray(z["ix_ele_lost"]), np.ascontiguousarray(z["ix_turn_lost"]))
    meta = {k: z[k] for k in z.files if k not in ("vec6", "beta", "state", "ix_ele_lost", "ix_turn_lost",
                                                   "next_turn")}
    return b, int(z["next_turn"]), meta
