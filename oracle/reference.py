"""The reference's own compiled code, for pinning the oracle.
TEST INFRASTRUCTURE ONLY.

``build_sparsity_reference`` calls build_sparsity_pattern_seq from the
reference's pyop2/sparsity_utils.cxx, compiled unmodified into
oracle/_ref/libref_sparsity.so by oracle/build.py.
"""

import ctypes as C

import numpy as np

from . import build as _build


class _Set(C.Structure):
    _fields_ = [("size", C.c_int), ("exec_size", C.c_int)]


class _Map(C.Structure):
    _fields_ = [("frm", C.POINTER(_Set)), ("to", C.POINTER(_Set)), ("dim", C.c_int),
                ("map", C.POINTER(C.c_int))]


def available():
    return _build.ref_lib_path() is not None


def build_sparsity_reference(rmult, cmult, nrows, maps):
    path = _build.ref_lib_path() or _build.build_ref()
    if path is None:
        raise RuntimeError("reference sparsity_utils.cxx is not available")
    lib = C.CDLL(path)
    keep = []
    n = len(maps)
    rarr, carr = (C.POINTER(_Map) * n)(), (C.POINTER(_Map) * n)()
    for k, (rm, cm) in enumerate(maps):
        for m, dst in ((rm, rarr), (cm, carr)):
            frm = _Set(m.iterset.size, 0)
            to = _Set(m.dataset.size, 0)
            vals = np.ascontiguousarray(m.values, np.int32)
            mm = _Map(C.pointer(frm), C.pointer(to), m.dim, vals.ctypes.data_as(C.POINTER(C.c_int)))
            keep += [frm, to, vals, mm]
            dst[k] = C.pointer(mm)
    nnz, rowptr, colidx = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_int)()
    nz = C.c_int()
    lib.build_sparsity_pattern_seq(rmult, cmult, nrows, n, rarr, carr, C.byref(nnz),
                                   C.byref(rowptr), C.byref(colidx), C.byref(nz))
    lsize = nrows * rmult
    libc = C.CDLL(None)
    out = (np.ctypeslib.as_array(rowptr, (lsize + 1,)).copy(),
           np.ctypeslib.as_array(colidx, (max(nz.value, 1),))[:nz.value].copy(),
           np.ctypeslib.as_array(nnz, (max(lsize, 1),))[:lsize].copy())
    for p in (nnz, rowptr, colidx):
        libc.free(C.cast(p, C.c_void_p))
    return out
