"""The reference's own compiled code, for pinning the oracle.
TEST INFRASTRUCTURE ONLY.

``build_sparsity_reference`` calls build_sparsity_pattern_seq from the
reference's pyop2/sparsity_utils.cxx, compiled unmodified into
oracle/_ref/libref_sparsity.so by oracle/build.py.

``plan_reference`` runs the reference's Plan (pyop2/plan.pyx, translated by
Cython and compiled by oracle/build.py) on a loop described by plain arrays
(see ``plan_case``).  The module imports ``base`` (for ``base.Dat`` /
``base.Mat`` isinstance tests) and ``utils.align``, and uses the Python 2
dict methods ``has_key`` / ``iterkeys`` of OrderedDict; it is imported with
stand-ins for those two modules and with an OrderedDict that has the two
methods, all put back once the import is done.  The module's ``numpy`` is
then a view of numpy whose ``unique`` returns a flat inverse, as numpy 1.x
did (numpy 2 gives it the input's shape, which ``inv[i::l]`` in
plan.pyx:151-152 would slice by rows).
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


# ---------------------------------------------------------------- Plan
_PLAN = {}


class _RefDat(object):
    pass


class _RefMat(object):
    pass


class _Obj(object):
    def __init__(self, **kw):
        self.__dict__.update(kw)


def _plan_module():
    if "mod" in _PLAN:
        return _PLAN["mod"]
    import collections
    import importlib.util
    import sys
    import types
    path = _build.ref_plan_path() or _build.build_ref_plan()
    if path is None:
        raise RuntimeError("reference plan.pyx is not available")

    class _Py2OrderedDict(collections.OrderedDict):
        def has_key(self, k):
            return k in self

        def iterkeys(self):
            return iter(self.keys())

    base = types.ModuleType("base")
    base.Dat, base.Mat = _RefDat, _RefMat
    utils = types.ModuleType("utils")
    # pyop2/utils.py align: round up to a multiple of the alignment
    utils.align = lambda nbytes, alignment=16: ((nbytes + alignment - 1) // alignment) * alignment
    saved = {k: sys.modules.get(k) for k in ("base", "utils")}
    odict = collections.OrderedDict
    sys.modules["base"], sys.modules["utils"] = base, utils
    collections.OrderedDict = _Py2OrderedDict
    try:
        spec = importlib.util.spec_from_file_location("plan", path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        collections.OrderedDict = odict
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    mod.numpy = _Numpy1Unique()
    _PLAN["mod"] = mod
    return mod


class _Numpy1Unique(object):
    """numpy, except that ``unique(..., return_inverse=True)`` returns the
    inverse flattened (the numpy 1.x result for a multi-dimensional input)."""

    def __getattr__(self, name):
        return getattr(np, name)

    @staticmethod
    def unique(ar, *a, **kw):
        r = np.unique(ar, *a, **kw)
        if kw.get("return_inverse") and kw.get("axis") is None:
            r = list(r)
            k = 2 if kw.get("return_index") else 1
            r[k] = np.asarray(r[k]).reshape(-1)
            r = tuple(r)
        return r


def plan_available():
    return _build.ref_plan_path() is not None


PLAN_FIELDS = ("nblocks", "nelems", "offset", "ind_map", "loc_map", "ind_sizes", "ind_offs",
               "nindirect", "nshared", "thrcol", "nthrcol", "ncolors", "ncolblk", "blkmap")


def plan_case(size, maps, dats, args, mats=None):
    """A loop for the plan builders, as plain data: ``size`` elements;
    ``maps`` {name: (values [size][dim] int32, target set size)}; ``dats``
    {name: (set size, numpy dtype, cdim)}; ``mats`` {name: row map name};
    ``args`` [(data name, map name or None, idx or None, access)] with access
    one of READ/WRITE/RW/INC (Mats: INC, map name = the row map)."""
    return dict(size=int(size), maps=maps, dats=dats, mats=mats or {}, args=list(args))


def plan_reference(case, partition_size, matrix_coloring=False, staging=True, thread_coloring=True):
    """{field: value} of the reference Plan built for ``case``."""
    mod = _plan_module()
    maps = {n: _Obj(values=np.ascontiguousarray(v, np.int32), dim=int(np.asarray(v).shape[1]),
                    dataset=_Obj(size=int(t)))
            for n, (v, t) in case["maps"].items()}
    data = {}
    for n, (ssize, dtype, cdim) in case["dats"].items():
        d = _RefDat()
        d.dataset, d.dtype, d.cdim = _Obj(size=int(ssize)), np.dtype(dtype), int(cdim)
        data[n] = d
    for n, rmap in case["mats"].items():
        m = _RefMat()
        m.sparsity = _Obj(maps=[(maps[rmap], maps[rmap])])
        data[n] = m
    rargs = []
    for name, mname, idx, access in case["args"]:
        is_mat = name in case["mats"]
        ind = mname is not None and idx is not None and not is_mat
        rargs.append(_Obj(data=data[name], map=maps[mname] if mname else None, idx=idx,
                          _is_mat=is_mat, _is_indirect=ind,
                          _is_indirect_reduction=ind and access == "INC"))
    p = mod.Plan(None, _Obj(size=case["size"]), *rargs, partition_size=partition_size,
                 matrix_coloring=matrix_coloring, staging=staging, thread_coloring=thread_coloring)
    return {f: (np.asarray(getattr(p, f)) if not isinstance(getattr(p, f), int) else getattr(p, f))
            for f in PLAN_FIELDS}
