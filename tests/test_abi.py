"""The C-ABI library: it loads, and exports every entry point that
include/op2b200.h declares (no device call is made).  CPU only."""

import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "op2b200.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^int\s+(op2b_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib():
    from pyop2_b200.csrc import build
    path = build.build()
    from pyop2_b200 import _lib
    return _lib.load(path), path


def test_library_loads_and_exports_all(lib):
    handle, path = lib
    names = declared()
    assert len(names) > 40
    for n in names:
        assert hasattr(handle, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (op2b_\w+)", out))
    assert set(names) == exported


def test_binding_declares_every_symbol(lib):
    from pyop2_b200 import _lib
    assert set(_lib.EXPORTED) == set(declared())


def test_calls_before_init_fail_cleanly(lib):
    import ctypes as C
    from pyop2_b200 import _lib
    p = C.c_uint64()
    rc = _lib._lib.op2b_malloc(C.byref(p), 16)
    assert rc != 0
    assert "op2b_init" in _lib.last_error()
