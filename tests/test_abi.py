"""The C-ABI library loads and exports every entry point include/hercules_b200.h
declares (no compute calls: runs without a GPU)."""
import ctypes
import os
import re

from hercules_b200 import build
from hercules_b200.engine import ABI_SYMBOLS, LIB_PATH

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "hercules_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(hc_[a-z_]+)\s*\(", txt)))


def test_header_matches_binding_list():
    assert declared_symbols() == sorted(ABI_SYMBOLS)


def test_library_exports_all_symbols():
    build.build()
    lib = ctypes.CDLL(LIB_PATH)
    for s in declared_symbols():
        assert hasattr(lib, s), s


def test_error_strings_without_gpu():
    lib = ctypes.CDLL(build.build())
    lib.hc_error_string.restype = ctypes.c_char_p
    assert lib.hc_error_string(-5) == b"NaN error"
    assert lib.hc_error_string(0) == b"ok"
