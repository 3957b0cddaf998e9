"""Extract the reference's golden vectors for the bmad_standard path into
tests/golden/*.json.  Reads the reference checkout given on the command line
as text; the JSON files are committed so tests never need the reference.

    python tests/golden/make_golden.py REFERENCE_ROOT

Sources (relative to the reference root):
  regression_tests/tracking_method_test/output.correct  ("<ELE>: Bmad_Standard" rows)
  regression_tests/fringe_test/output.correct           (Hwang edge kick deltas)
  regression_tests/aperture_test/output.correct         (aperture states, unstable factors)
  regression_tests/multipole_test/output.correct        ("MULT-<tilt><kicks>-<ELE>" rows: multipole_ele_to_ab)
  regression_tests/coord_test/output.correct            (offset_particle set / unset, forward rows of the
                                                         misaligned solenoid and bends)
"""
import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def parse_line(line):
    m = re.match(r'\s*"([^"]+)"\s+(ABS|REL|STR|VEC_REL)\s+(\S+)\s+(.*)$', line)
    if not m:
        return None
    name, kind, tol, rest = m.groups()
    vals = rest.split()
    return name, kind, float(tol) if kind != "STR" else tol, vals


def main(ref: Path):
    out = {}
    tm = (ref / "regression_tests/tracking_method_test/output.correct").read_text().splitlines()
    rows = {}
    for line in tm:
        p = parse_line(line)
        if not p:
            continue
        name, kind, tol, vals = p
        if not name.endswith(": Bmad_Standard") or "-" in name.split(":")[0]:
            continue
        rows[name.split(":")[0]] = {"tol": tol, "values": [float(v) for v in vals], "text": vals}
    out["tracking_method"] = rows
    # the same rows tracked with absolute time (bmad_com%absolute_time_tracking
    # = T; tracking_method_test.f90:113-119,174-179: elements with time-varying
    # fields only)
    abs_rows = {}
    for line in tm:
        p = parse_line(line)
        if not p:
            continue
        name, kind, tol, vals = p
        head = name.split(":")[0]
        if name.endswith(": Bmad_Standard") and head.endswith("-Abs_Time"):
            abs_rows[head[:-len("-Abs_Time")]] = {"tol": tol, "values": [float(v) for v in vals], "text": vals}
    out["tracking_method_abs_time"] = abs_rows
    fr = {}
    for line in (ref / "regression_tests/fringe_test/output.correct").read_text().splitlines():
        p = parse_line(line)
        if p and p[0] in ("Up-Orb", "Dn-Orb"):
            fr[p[0]] = {"tol": p[2], "values": [float(v) for v in p[3]], "text": p[3]}
    out["fringe"] = fr
    ap = {}
    for line in (ref / "regression_tests/aperture_test/output.correct").read_text().splitlines():
        p = parse_line(line)
        if p and re.match(r"(EC|RC)_[SU]_", p[0]):
            ap[p[0]] = {"tol": p[2], "values": [float(v) for v in p[3]], "text": p[3]}
    out["aperture"] = ap
    mp = {}
    for line in (ref / "regression_tests/multipole_test/output.correct").read_text().splitlines():
        p = parse_line(line)
        if p and re.match(r"MULT-[12][12]-(QQ|BB|MM|EE)$", p[0]):
            mp[p[0]] = {"tol": p[2], "values": [float(v) for v in p[3][:6]], "ix": int(p[3][6]), "text": p[3][:6]}
    out["multipole"] = mp
    co = {}
    for line in (ref / "regression_tests/coord_test/output.correct").read_text().splitlines():
        p = parse_line(line)
        if p and re.match(r"(Q1|B0|B1|B2):O:1:D:1:.*-orb$", p[0]):
            co[p[0]] = {"tol": p[2], "values": [float(v) for v in p[3]], "text": p[3]}
    out["coord"] = co
    (HERE / "reference_golden.json").write_text(json.dumps(out, indent=1, sort_keys=True))
    print(f"tracking_method rows: {len(rows)} (+{len(abs_rows)} in absolute time), fringe rows: {len(fr)}, "
          f"aperture rows: {len(ap)}, "
          f"multipole rows: {len(mp)}, coord rows: {len(co)}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py REFERENCE_ROOT")
    main(Path(sys.argv[1]))
