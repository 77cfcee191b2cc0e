"""The C ABI library loads and exports every symbol include/*.h declares
(no device call is made: these run without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            src = open(os.path.join(inc, f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(sb2_\w+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    from seldon_b200 import _lib
    lib = _lib.load()
    declared = _declared()
    assert len(declared) >= 25
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing


def test_python_prototypes_cover_header():
    from seldon_b200 import _lib
    assert _declared() <= set(_lib.exported_names())


def test_status_strings_without_gpu():
    from seldon_b200 import _lib
    lib = _lib.load()
    assert lib.sb2_status_string(0) == b"ok"
    assert b"CSR" in lib.sb2_status_string(_lib.SB2_ERR_INVALID_CSR)
    assert lib.sb2_version() >= 10000
