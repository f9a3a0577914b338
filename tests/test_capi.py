"""The C-ABI library builds for sm_100a, loads, and exports every entry point
declared in include/dalia_bta.h (no GPU needed)."""
import os
import re

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdrs = [os.path.join(REPO, "include", f) for f in os.listdir(os.path.join(REPO, "include"))
            if f.endswith(".h")]
    names = set()
    for h in hdrs:
        txt = open(h).read()
        names |= set(re.findall(r"^\s*(?:int|size_t|const char\*)\s+(bta_\w+)\s*\(", txt, re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("bta_create", "bta_pobtaf", "bta_pobtas", "bta_pobtasi", "bta_logdet"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from dalia_b200 import _lib
    from dalia_b200.build import build

    build()
    lib = _lib.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert lib.bta_error_string(3).decode() == "matrix is not positive definite"


def test_python_binding_covers_header():
    from dalia_b200 import _lib

    assert set(declared_symbols()) <= set(_lib.SIGNATURES)
