"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute calls: runs without a GPU)."""
import ctypes
import re
from pathlib import Path

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
    # bgt_element: 12 int32 + 35 doubles + 6 x 22 doubles
    assert ctypes.sizeof(_lib.BgtElement) == 12 * 4 + 35 * 8 + 6 * 22 * 8
    assert ctypes.sizeof(_lib.BgtSpecies) == 24
    assert ctypes.sizeof(_lib.BgtTuning) == 20
