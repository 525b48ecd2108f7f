"""The C-ABI library: it loads and exports every entry point include/champ_b200.h declares
(no compute calls, so this runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "champ_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(champ_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    from champ_b200 import build
    build.build()
    return ctypes.CDLL(build.LIB)


def test_library_exports_every_declared_symbol(lib):
    syms = header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), s


def test_binding_lists_match_header():
    from champ_b200.engine import EXPORTED_SYMBOLS
    assert sorted(EXPORTED_SYMBOLS) == header_symbols()


def test_version_string(lib):
    lib.champ_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.champ_version()


def test_errors_are_returned_not_raised(lib):
    lib.champ_create.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]
    lib.champ_last_error.restype = ctypes.c_char_p
    out = ctypes.c_void_p()
    rc = lib.champ_create(None, 10, 0, None, ctypes.byref(out))
    assert rc == 1 and b"null" in lib.champ_last_error()
