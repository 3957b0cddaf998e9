"""Bmad lattice files and long_term_tracking inputs for the tracker's lattices.

* ``write_lattice``: a :class:`bgt.lattice.Lattice` as a Bmad lattice file
  (``name: key, attr = value, ...`` element definitions, one line, ``use``),
  with every real attribute written to 17 significant digits so that Bmad
  reads back the same doubles.  Together with ``write_ltt_init`` (a
  long_term_tracking ``&params`` namelist, BEAM mode, ``bmad_standard``) and
  a beam file from ``bgt.beam_io.write_ascii_beam`` it is the lattice's twin
  for a machine with Bmad installed: the reference's own tracking of the same
  lattice and particles (bsim/modules/lt_tracking_mod.f90, ltt_params_struct
  :40-99 for the parameter names).
* ``read_lattice``: the subset of the Bmad lattice language those files and
  the reference's element tests use -- element definitions (with
  inheritance from an earlier element, ``name[attr] = value`` settings, flag
  attributes such as a bare ``tilt``), ``parameter[...]``, one ``line`` and
  ``use`` -- with arithmetic expressions in ``pi``, ``twopi`` and the
  physical constants.  It follows the parser's conventions where the tracker
  depends on them (bmad/parsing/parser_set_attribute_mod.f90:1762-1800 for
  flag attributes; an rbend's ``l`` is its chord, as :func:`bgt.lattice.
  rbend_to_sbend` converts it).

Element attribute names are Bmad's own (``ele%value`` names, ``a<n>`` /
``b<n>`` / ``a<n>_elec`` / ``b<n>_elec`` multipoles, ``k<n>l`` / ``k<n>sl`` /
``t<n>`` for a thin multipole), kept alike so that the files need no
translation on either side.
"""
from __future__ import annotations

import ast
import math
import operator
import re
from pathlib import Path
from typing import Dict, List, Optional, Tuple

from . import lattice as L

_END_NAMES = ("entrance_end", "exit_end", "both_ends", "no_end")
_FRINGE_NAMES = ("none", "basic_bend", "full", "hard_edge_only", "soft_edge_only", "sad_full", "linear_edge")
_APERTURE_NAMES = ("rectangular", "elliptical")
_SPECIES = {"electron": (L.M_ELECTRON, -1), "positron": (L.M_ELECTRON, 1),
            "proton": (938.27208816e6, 1), "antiproton": (938.27208816e6, -1)}
# sim_utils/interfaces/physical_constants.f90
_CONSTANTS = {"pi": math.pi, "twopi": 2 * math.pi, "c_light": 2.99792458e8, "m_electron": L.M_ELECTRON,
              "m_proton": 938.27208816e6, "e_charge": 1.602176634e-19, "degrees": math.pi / 180}
_REALS = [n for n in L._VALUE_NAMES if n not in ("p0c", "e_tot")]


def _fmt(v: float) -> str:
    s = repr(float(v))
    return s if ("e" in s or "." in s or "inf" in s or "nan" in s) else s + ".0"


# ---------------------------------------------------------------------------
# writing

def _element_attrs(e: L.Element) -> List[str]:
    out = []
    for n in _REALS:
        v = e.values.get(n)
        if v is None or (v == 0 and n != "l"):
            continue
        if n == "ds_step" and e.user_ds_step == 0:
            continue  # filled in by the bookkeeper, not given by the user
        out.append(f"{n} = {_fmt(v)}")
    steps = e.user_num_steps if e.user_num_steps is not None else e.num_steps
    if steps:
        out.append(f"num_steps = {int(steps)}")
    if not e.is_on:
        out.append("is_on = F")
    default_fringe = {"sbend": "basic_bend", "rfcavity": "full"}.get(e.key, "none")
    if e.fringe_type != default_fringe:
        out.append(f"fringe_type = {e.fringe_type}")
    if e.fringe_at != "both_ends":
        out.append(f"fringe_at = {e.fringe_at}")
    default_ap = "elliptical" if e.key == "ecollimator" else "rectangular"
    if e.aperture_type != default_ap:
        out.append(f"aperture_type = {e.aperture_type}")
    if e.aperture_at != "exit_end":
        out.append(f"aperture_at = {e.aperture_at}")
    if e.offset_moves_aperture != (e.key in ("rcollimator", "ecollimator")):
        out.append(f"offset_moves_aperture = {'T' if e.offset_moves_aperture else 'F'}")
    if not e.scale_multipoles:
        out.append("scale_multipoles = F")
    if e.key == "rfcavity" and e.coupler_at != "exit_end":
        out.append(f"coupler_at = {e.coupler_at}")
    if e.key == "multipole":
        for n, v in sorted(e.a_pole.items()):
            out.append(f"k{n}l = {_fmt(v)}")
        for n, v in sorted(e.ksl_pole.items()):
            out.append(f"k{n}sl = {_fmt(v)}")
        for n, v in sorted(e.b_pole.items()):
            out.append(f"t{n} = {_fmt(v)}")
    else:
        for n, v in sorted(e.a_pole.items()):
            out.append(f"a{n} = {_fmt(v)}")
        for n, v in sorted(e.b_pole.items()):
            out.append(f"b{n} = {_fmt(v)}")
    for n, v in sorted(e.a_pole_elec.items()):
        out.append(f"a{n}_elec = {_fmt(v)}")
    for n, v in sorted(e.b_pole_elec.items()):
        out.append(f"b{n}_elec = {_fmt(v)}")
    return out


def _bmad_name(name: str) -> str:
    s = re.sub(r"[^A-Za-z0-9_.]", "_", name or "E")
    if not s[0].isalpha():
        s = "E" + s
    return s[:36]


def write_lattice(lat: L.Lattice, path: str, geometry: str = "closed", line_name: str = "ring") -> None:
    """The lattice as a Bmad lattice file.  Elements that share a name and
    all attributes are written once and repeated in the line; elements that
    share a name but differ (error variants) get a numbered name each."""
    defs: Dict[str, Tuple[str, str]] = {}
    seq: List[str] = []
    for e in lat.elements:
        attrs = ", ".join([e.key] + _element_attrs(e))
        base = _bmad_name(e.name).upper()
        name = base
        k = 1
        while name in defs and defs[name][1] != attrs:
            k += 1
            name = f"{base}_{k}"
        defs.setdefault(name, (e.key, attrs))
        seq.append(name)
    lines = [f"! {lat.name or 'lattice'}: {len(lat.elements)} elements, written by bgt.bmad_twin",
             f"parameter[geometry] = {geometry}",
             f"parameter[particle] = {lat.species.name}",
             f"parameter[e_tot] = {_fmt(lat.e_tot)}",
             ""]
    for name, (_, attrs) in defs.items():
        lines.append(f"{name}: {attrs}")
    lines.append("")
    items = ", ".join(seq)
    # wrap the line at about 100 characters: a trailing comma continues it
    wrapped, cur = [], f"{line_name}: line = ("
    for tok in items.split(", "):
        if len(cur) + len(tok) > 100:
            wrapped.append(cur)
            cur = "  "
        cur += tok + ", "
    wrapped.append(cur[:-2] + ")")
    lines.extend(wrapped)
    lines.append(f"use, {line_name}")
    Path(path).write_text("\n".join(lines) + "\n")


def write_ltt_init(path: str, lat_file: str, beam_file: str, n_turns: int, beam_output_file: str = "beam_out.dat",
                   aperture_limit_on: bool = True) -> None:
    """A long_term_tracking input (``&params`` namelist) tracking the beam
    file through the lattice with bmad_standard, BEAM mode, no radiation,
    spin or ramping, relative RF time -- the tracker's model of the path."""
    t = "T" if aperture_limit_on else "F"
    text = f"""&params
  ltt%lat_file = '{lat_file}'
  ltt%simulation_mode = 'BEAM'
  ltt%tracking_method = 'BMAD'
  ltt%n_turns = {int(n_turns)}
  ltt%beam_output_file = '{beam_output_file}'
  ltt%beam_output_every_n_turns = {int(n_turns)}
  ltt%add_closed_orbit_to_init_position = F
  ltt%rfcavity_on = T
  beam_init%position_file = '{beam_file}'
  bmad_com%radiation_damping_on = F
  bmad_com%radiation_fluctuations_on = F
  bmad_com%spin_tracking_on = F
  bmad_com%absolute_time_tracking = F
  bmad_com%aperture_limit_on = {t}
/
"""
    Path(path).write_text(text)


# ---------------------------------------------------------------------------
# reading

_BINOPS = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul, ast.Div: operator.truediv,
           ast.Pow: operator.pow}


def _eval(expr: str, names: Dict[str, float]) -> float:
    """An arithmetic expression in numbers, names and + - * / ** / ^."""
    tree = ast.parse(expr.strip().replace("^", "**"), mode="eval")

    def ev(n):
        if isinstance(n, ast.Expression):
            return ev(n.body)
        if isinstance(n, ast.Constant) and isinstance(n.value, (int, float)):
            return float(n.value)
        if isinstance(n, ast.Name):
            key = n.id.lower()
            if key in names:
                return names[key]
            if key in _CONSTANTS:
                return _CONSTANTS[key]
            raise ValueError(f"unknown name {n.id!r} in {expr!r}")
        if isinstance(n, ast.UnaryOp) and isinstance(n.op, (ast.USub, ast.UAdd)):
            v = ev(n.operand)
            return -v if isinstance(n.op, ast.USub) else v
        if isinstance(n, ast.BinOp) and type(n.op) in _BINOPS:
            return _BINOPS[type(n.op)](ev(n.left), ev(n.right))
        raise ValueError(f"unsupported expression {expr!r}")

    return ev(tree)


def _split_top(s: str, sep: str = ",") -> List[str]:
    out, depth, cur = [], 0, []
    for ch in s:
        if ch in "({[":
            depth += 1
        elif ch in ")}]":
            depth -= 1
        if ch == sep and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    out.append("".join(cur))
    return [x.strip() for x in out]


def _statements(text: str) -> List[str]:
    stmts, cur = [], ""
    for raw in text.splitlines():
        line = raw.split("!", 1)[0].rstrip()
        if not line.strip():
            continue
        cur = (cur + " " + line.strip()) if cur else line.strip()
        if cur.endswith("&"):
            cur = cur[:-1]
            continue
        if cur.endswith(",") or cur.count("(") > cur.count(")"):
            continue
        stmts.append(cur)
        cur = ""
    if cur:
        stmts.append(cur)
    return stmts


def _set_attr(d: dict, key: str, attr: str, val: Optional[str], names: Dict[str, float]) -> None:
    a = attr.lower()
    if val is None:
        # flag attributes (parser_set_attribute_mod.f90:1762-1800)
        m = re.fullmatch(r"t(\d+)", a)
        if key == "multipole" and m:
            n = int(m.group(1))
            d["b_pole"][n] = math.pi / (2 * n + 2)
        elif a == "tilt":
            t = {"quadrupole": 4.0, "sextupole": 6.0, "octupole": 8.0}.get(key)
            if t is None:
                raise ValueError(f"no default tilt for a {key}")
            d["values"]["tilt"] = math.pi / t
        elif a in ("fint", "fintx") and key in ("sbend", "rbend"):
            d["values"][a] = 0.5
        else:
            raise ValueError(f"attribute {attr!r} needs a value")
        return
    v = val.strip()
    low = v.lower()
    if a in ("fringe_type",):
        if low not in _FRINGE_NAMES:
            raise ValueError(f"fringe_type {v!r} is not one the tracker knows")
        d["fringe_type"] = low
    elif a in ("fringe_at", "aperture_at", "coupler_at"):
        if low not in _END_NAMES:
            raise ValueError(f"{attr} {v!r}")
        d[a] = low
    elif a == "aperture_type":
        if low not in _APERTURE_NAMES:
            raise ValueError(f"aperture_type {v!r}")
        d["aperture_type"] = low
    elif a in ("offset_moves_aperture", "is_on", "scale_multipoles"):
        d[a] = low in ("t", "true", ".true.")
    elif a == "exact_multipoles":
        d["exact_multipoles"] = 0 if low == "off" else (1 if low == "vertically_pure" else 2)
    elif a == "num_steps":
        d["num_steps"] = int(round(_eval(v, names)))
    elif a in ("x_limit", "y_limit"):
        x = _eval(v, names)
        d["values"][a[0] + "1_limit"] = x
        d["values"][a[0] + "2_limit"] = x
    elif a == "aperture":
        x = _eval(v, names)
        for n in ("x1_limit", "x2_limit", "y1_limit", "y2_limit"):
            d["values"][n] = x
    elif a in ("cavity_type", "tracking_method", "mat6_calc_method", "field_calc", "type", "alias", "descrip"):
        pass  # no effect on bmad_standard tracking of the elements the tracker supports
    else:
        num = _eval(v, names)
        m = re.fullmatch(r"([ab])(\d+)(_elec)?", a)
        mk = re.fullmatch(r"k(\d+)(s?)l", a)
        mt = re.fullmatch(r"t(\d+)", a)
        if m and key not in ("multipole",):
            arr = ("a_pole" if m.group(1) == "a" else "b_pole") + ("_elec" if m.group(3) else "")
            d[arr][int(m.group(2))] = num
        elif mk and key == "multipole":
            d["ksl_pole" if mk.group(2) else "a_pole"][int(mk.group(1))] = num
        elif mt and key == "multipole":
            d["b_pole"][int(mt.group(1))] = num
        else:
            d["values"][a] = num


def _new_def(key: str) -> dict:
    return {"key": key, "values": {}, "num_steps": 0, "is_on": True, "fringe_type": None, "fringe_at": "both_ends",
            "aperture_type": None, "aperture_at": "exit_end", "offset_moves_aperture": None,
            "exact_multipoles": 0, "scale_multipoles": True, "a_pole": {}, "b_pole": {}, "ksl_pole": {},
            "a_pole_elec": {}, "b_pole_elec": {}, "coupler_at": "exit_end"}


def _copy_def(d: dict) -> dict:
    out = dict(d)
    for k in ("values", "a_pole", "b_pole", "ksl_pole", "a_pole_elec", "b_pole_elec"):
        out[k] = dict(d[k])
    return out


def read_lattice(path_or_text: str, text: bool = False) -> L.Lattice:
    """A Bmad lattice file (the subset described in the module docstring)
    as a finalized :class:`bgt.lattice.Lattice`."""
    src = path_or_text if text else Path(path_or_text).read_text()
    defs: Dict[str, dict] = {}
    lines: Dict[str, List[str]] = {}
    params: Dict[str, str] = {}
    names: Dict[str, float] = {}
    use = None
    for st in _statements(src):
        low = st.lower()
        m = re.fullmatch(r"(parameter|beginning|particle_start)\[(\w+)\]\s*=\s*(.+)", st, re.I)
        if m:
            params[f"{m.group(1).lower()}[{m.group(2).lower()}]"] = m.group(3).strip()
            continue
        m = re.fullmatch(r"use\s*,\s*(\w+)", st, re.I)
        if m:
            use = m.group(1).lower()
            continue
        m = re.fullmatch(r"([\w.]+)\[(\w+)\]\s*=\s*(.+)", st)
        if m:
            name = m.group(1).lower()
            if name not in defs:
                raise ValueError(f"{m.group(1)} is not defined")
            _set_attr(defs[name], defs[name]["key"], m.group(2), m.group(3), names)
            continue
        m = re.fullmatch(r"([\w.]+)\s*:\s*line\s*=\s*\((.*)\)", st, re.I)
        if m:
            lines[m.group(1).lower()] = [x.lower() for x in _split_top(m.group(2)) if x]
            continue
        m = re.fullmatch(r"([\w.]+)\s*:\s*(.+)", st)
        if m:
            name = m.group(1).lower()
            parts = _split_top(m.group(2))
            head = parts[0].lower()
            if head in defs:
                d = _copy_def(defs[head])
            elif head in L.KEYS or head == "rbend":
                d = _new_def(head)
            else:
                raise ValueError(f"{st!r}: unknown element type or base element {parts[0]!r}")
            for p in parts[1:]:
                if "=" in p:
                    k, v = p.split("=", 1)
                    _set_attr(d, d["key"], k.strip(), v, names)
                else:
                    _set_attr(d, d["key"], p.strip(), None, names)
            defs[name] = d
            continue
        m = re.fullmatch(r"(\w+)\s*=\s*(.+)", st)
        if m and low.split("=")[0].strip() not in defs:
            names[m.group(1).lower()] = _eval(m.group(2), names)
            continue
        raise ValueError(f"cannot read the statement {st!r}")
    if use is None:
        if len(lines) != 1:
            raise ValueError("no 'use' statement")
        use = next(iter(lines))
    if use not in lines:
        raise ValueError(f"line {use!r} is not defined")

    def expand(item: str, depth: int = 0) -> List[str]:
        if depth > 20:
            raise ValueError("line nesting too deep")
        if item in lines:
            return [x for it in lines[item] for x in expand(it, depth + 1)]
        return [item]

    eles = []
    for nm in expand(use):
        if nm not in defs:
            raise ValueError(f"element {nm!r} in the line is not defined")
        d = defs[nm]
        e = L.Element(d["key"], nm.upper(), dict(d["values"]), num_steps=d["num_steps"], is_on=d["is_on"],
                      fringe_type=d["fringe_type"], fringe_at=d["fringe_at"], aperture_type=d["aperture_type"],
                      aperture_at=d["aperture_at"], offset_moves_aperture=d["offset_moves_aperture"],
                      exact_multipoles=d["exact_multipoles"], scale_multipoles=d["scale_multipoles"],
                      a_pole=dict(d["a_pole"]), b_pole=dict(d["b_pole"]), ksl_pole=dict(d["ksl_pole"]),
                      a_pole_elec=dict(d["a_pole_elec"]), b_pole_elec=dict(d["b_pole_elec"]),
                      coupler_at=d["coupler_at"])
        eles.append(e)
    sp_name = params.get("parameter[particle]", "positron").lower()
    if sp_name not in _SPECIES:
        raise ValueError(f"particle {sp_name!r}")
    mass, charge = _SPECIES[sp_name]
    species = L.Species(sp_name, mass, charge)
    if "parameter[e_tot]" in params:
        e_tot = _eval(params["parameter[e_tot]"], names)
        p0c = L.p0c_from_e_tot(e_tot, mass)
    elif "parameter[p0c]" in params:
        p0c = _eval(params["parameter[p0c]"], names)
        e_tot = math.sqrt(p0c * p0c + mass * mass)
    else:
        raise ValueError("parameter[e_tot] or parameter[p0c] is required")
    lat = L.Lattice(eles, species, p0c, e_tot, use)
    return lat.finalize()


# ---------------------------------------------------------------------------
# a complete twin

def write_twin(lat: L.Lattice, vec6, out_dir: str, n_turns: int, name: str = "ring",
               geometry: str = "closed") -> Dict[str, str]:
    """Lattice file, beam file (the particles ``vec6[6, n]``, alive, at the
    start of the lattice) and long_term_tracking input in ``out_dir``: run
    ``long_term_tracking <name>.init`` there with Bmad to track the same
    particles through the same lattice with the reference."""
    import numpy as np

    from . import beam_io
    from .track import Bunch

    out = Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    files = {"lattice": str(out / f"{name}.bmad"), "beam": str(out / f"{name}_beam.dat"),
             "init": str(out / f"{name}.init")}
    write_lattice(lat, files["lattice"], geometry=geometry, line_name=name)
    b = Bunch.from_vec(np.asarray(vec6, dtype=np.float64), lat.p0c, lat.species.mass)
    beam_io.write_ascii_beam(files["beam"], [beam_io.BeamBunch.from_bunch(b, lat.p0c, lat.species.name)])
    write_ltt_init(files["init"], Path(files["lattice"]).name, Path(files["beam"]).name, n_turns,
                   beam_output_file=f"{name}_beam_out.dat")
    return files


def main(argv=None) -> None:
    """``python -m bgt.bmad_twin OUT_DIR [N_PARTICLES] [N_TURNS]``: the twin of
    the 64-cell ring with apertures and a sample of its matched beam (the
    particle-throughput benchmark's lattice and beam)."""
    import sys

    from . import rings

    args = list(sys.argv[1:] if argv is None else argv)
    if not args:
        raise SystemExit(main.__doc__)
    n = int(args[1]) if len(args) > 1 else 1000
    turns = int(args[2]) if len(args) > 2 else 1000
    lat = rings.fodo_ring(apertures=True)
    spec = rings.CONFIG1_BEAM
    v0 = rings.gaussian_beam(rings.BeamSpec(n, spec.emit_x, spec.emit_y, spec.sigma_z, spec.sigma_pz, spec.seed))
    for k, v in write_twin(lat, v0, args[0], turns).items():
        print(f"{k}: {v}")


if __name__ == "__main__":
    main()
