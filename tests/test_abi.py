"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import re
import shutil
import subprocess
from pathlib import Path

import pytest

from bgt import _lib

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    src = "\n".join(p.read_text() for p in sorted((ROOT / "include").glob("*.h")))
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|const char\*)\s+(bgt_\w+)\s*\(", src, re.M)))


def test_header_symbols_listed():
    assert declared_symbols() == sorted(_lib.EXPORTED)


def test_library_loads_and_exports():
    lib = _lib.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name
        assert isinstance(getattr(lib, name), ctypes._CFuncPtr)


def test_struct_layout_matches_header():
    # bgt_element: 12 int32 + 35 doubles + 6 x 22 doubles + 4 doubles + 8
    # collimator limits + 2 reference times
    assert ctypes.sizeof(_lib.BgtElement) == 12 * 4 + 35 * 8 + 6 * 22 * 8 + 4 * 8 + 8 * 8 + 2 * 8
    assert ctypes.sizeof(_lib.BgtSpecies) == 32
    assert ctypes.sizeof(_lib.BgtTuning) == 28


def test_struct_offsets_match_the_c_compiler(tmp_path):
    """The ctypes mirrors against the header as a C compiler lays it out."""
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    checks = {"bgt_element": (_lib.BgtElement, [f for f, _ in _lib.BgtElement._fields_]),
              "bgt_species": (_lib.BgtSpecies, [f for f, _ in _lib.BgtSpecies._fields_]),
              "bgt_tuning": (_lib.BgtTuning, [f for f, _ in _lib.BgtTuning._fields_])}
    lines = ['#include <stddef.h>', '#include <stdio.h>', f'#include "{ROOT / "include" / "bgt.h"}"',
             "int main(void) {"]
    for st, (_, fields) in checks.items():
        lines.append(f'  printf("{st} sizeof %zu\\n", sizeof({st}));')
        for f in fields:
            lines.append(f'  printf("{st} {f} %zu\\n", offsetof({st}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([gcc, "-o", str(exe), str(src)], check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {(a, b): int(c) for a, b, c in (ln.split() for ln in out if ln)}
    for st, (cls, fields) in checks.items():
        assert got[(st, "sizeof")] == ctypes.sizeof(cls), st
        for f in fields:
            assert got[(st, f)] == getattr(cls, f).offset, (st, f)


def _fortran_type_fields(src: str, name: str):
    """(field, kind, count) in declaration order of a bind(c) derived type
    of the Fortran shim."""
    body = re.search(rf"type, bind\(c\) :: {name}\n(.*?)\nend type", src, re.S).group(1)
    out = []
    for line in body.splitlines():
        m = re.match(r"\s*(integer\(c_int32_t\)|real\(c_double\))\s*::\s*(.*)$", line)
        if not m:
            continue
        kind = "i32" if "int32" in m.group(1) else "f64"
        for f in re.split(r",\s*(?![^()]*\))", m.group(2)):
            fm = re.match(r"(\w+)(?:\((\w+)\))?", f.strip())
            out.append((fm.group(1), kind, 22 if fm.group(2) else 1))
    return out


def test_fortran_shim_mirrors_the_c_structs_and_symbols():
    """The Fortran module (no compiler for it here) declares the C structs
    field for field in the header's order and binds only exported symbols."""
    import ctypes as C

    src = (ROOT / "bmad-ecosystem_b200" / "fortran" / "bgt_mod.f90").read_text()
    for fname, cls in (("bgt_element_c", _lib.BgtElement), ("bgt_species_c", _lib.BgtSpecies),
                       ("bgt_tuning_c", _lib.BgtTuning)):
        want = []
        for f, t in cls._fields_:
            if issubclass(t, C.Array):
                want.append((f, "f64", t._length_))
            else:
                want.append((f, "i32" if t is C.c_int32 else "f64", 1))
        assert _fortran_type_fields(src, fname) == want, fname
    bound = set(re.findall(r"bind\(c, name='(bgt_\w+)'\)", src))
    assert bound and bound <= set(declared_symbols())
