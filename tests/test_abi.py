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


@pytest.mark.parametrize("name", ["op2b_mat_zero_rows", "op2b_mat_zero_rows_static"])
def test_zero_rows_rejects_bad_rows_on_the_host(lib, name):
    """A listed row outside [0, mat_rows), or an element size other than 4 or
    8, is rejected before the library touches the device: the check runs even
    here, with no GPU and no op2b_init, and the device pointers (all 0) are
    never used."""
    import ctypes as C
    import numpy as np
    from pyop2_b200 import _lib
    fn = getattr(_lib._lib, name)
    for rows, elem_bytes, what in (([0, 3, 10], 8, "row 10"), ([-1], 8, "row -1"),
                                   ([2], 2, "elem_bytes 2")):
        r = np.asarray(rows, dtype=np.int32)
        rc = fn(0, 0, 0, 10, r.ctypes.data_as(C.POINTER(C.c_int32)), r.size, 1.0, elem_bytes, 0)
        assert rc == 3, (rows, rc)       # OP2B_ERR_ARG
        assert what in _lib.last_error()
