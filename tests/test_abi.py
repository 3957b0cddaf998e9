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
    # bgt_element: 12 int32 + 35 doubles + 6 x 22 doubles + 4 doubles
    assert ctypes.sizeof(_lib.BgtElement) == 12 * 4 + 35 * 8 + 6 * 22 * 8 + 4 * 8 + 8 * 8
    assert ctypes.sizeof(_lib.BgtSpecies) == 24
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
