"""CPU oracle: the reference's sequential backend, restated.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of bench.py as the checker; never by the B200 backend.

A minimal op2-shaped API (Set, Map, Dat, Global, Const, Kernel, Sparsity,
Mat, par_loop, IdentityMap, i, access modes) whose ``par_loop`` does what
pyop2/sequential.py + pyop2/host.py do:

* generate a C wrapper around the user kernel with the element loop of
  sequential.py:55-72 (vec-map pointer arrays, itspace loops, local tensor
  zeroed per entry, kernel call, vector-field addto inside the loops,
  scalar-field block addto after them) and the per-argument expressions of
  host.py:91-207;
* compile it with gcc (the reference used instant + mpicc, host.py:225-261);
* run it over [0, size) in element order (single rank: core = owned = exec,
  sequential.py:76-121), so INC args accumulate straight into the Dat in
  element order and Global args are updated in place;
* Mat insertion is PETSc's MatSetValuesLocal ADD/INSERT restated on a fixed
  CSR pattern (oracle_core.c), with addto_scalar skipping exact zeros when
  adding (mat_utils.cxx:10).

``openmp=True`` in :func:`par_loop` runs the restated OpenMP backend instead
(openmp.py:130-261): blocks of 1024 elements coloured with matrix colouring
(plan.pyx restated in :mod:`oracle.plan`), colours in order, the blocks of a
colour in parallel, per-thread Global reduction copies.
"""

import ctypes as C
import hashlib
import os
import subprocess
import tempfile

import numpy as np

from . import build as _build

_CORE = None


def core():
    global _CORE
    if _CORE is None:
        _CORE = C.CDLL(_build.build_oracle())
        _CORE.oracle_build_sparsity.restype = C.c_int
        _CORE.oracle_plan_color.restype = None
    return _CORE


# ------------------------------------------------------------------- API
class Access(object):
    def __init__(self, mode):
        self._mode = mode

    def __repr__(self):
        return "Access(%r)" % self._mode


READ, WRITE, RW, INC, MIN, MAX = (Access(m) for m in ("READ", "WRITE", "RW", "INC", "MIN", "MAX"))

_CTYPES = {"uint8": "unsigned char", "int8": "char", "int16": "short", "uint16": "unsigned short",
           "int32": "int", "uint32": "unsigned int", "int64": "long long",
           "uint64": "unsigned long long", "float32": "float", "float64": "double",
           "bool": "unsigned char"}


class Set(object):
    def __init__(self, size, dim=1, name=None):
        self.size = int(size)
        self.dim = tuple(np.atleast_1d(dim).astype(int).tolist())
        self.cdim = int(np.prod(self.dim))
        self.name = name

    def __call__(self, *extents):
        return IterationSpace(self, extents)


class IterationSpace(object):
    def __init__(self, iterset, extents):
        self.iterset = iterset
        self.extents = tuple(int(e) for e in extents)


class IterationIndex(object):
    def __init__(self, index=None):
        self.index = index

    def __getitem__(self, k):
        return IterationIndex(k)


i = IterationIndex()


class Arg(object):
    def __init__(self, data=None, map=None, idx=None, access=None):
        self.data, self.map, self.idx, self.access = data, map, idx, access


class Map(object):
    def __init__(self, iterset, dataset, dim, values, name=None):
        self.iterset, self.dataset, self.dim = iterset, dataset, int(dim)
        self.values = np.ascontiguousarray(np.asarray(values, dtype=np.int32).reshape(iterset.size, self.dim))
        self.name = name

    def __getitem__(self, idx):
        return Arg(map=self, idx=idx)


IdentityMap = Map(Set(0), Set(0), 1, np.zeros(0, np.int32), "identity")


class Dat(object):
    def __init__(self, dataset, data=None, dtype=None, name=None, soa=False):
        if data is None:
            data = np.zeros(dataset.size * dataset.cdim, dtype=dtype or np.float64)
        self.dataset = dataset
        self.data = np.ascontiguousarray(np.array(data, dtype=dtype).reshape((dataset.size,) + dataset.dim))
        self.cdim = dataset.cdim
        self.soa = soa
        self.name = name

    @property
    def ctype(self):
        return _CTYPES[self.data.dtype.name]

    def __call__(self, path, access):
        if isinstance(path, Map):
            return Arg(self, path, None, access)
        path.data, path.access = self, access
        return path


class Global(object):
    def __init__(self, dim, data=None, dtype=None, name=None):
        self.dim = tuple(np.atleast_1d(dim).astype(int).tolist())
        self.cdim = int(np.prod(self.dim))
        self.data = np.ascontiguousarray(np.array(data, dtype=dtype).reshape(self.dim))
        self.name = name

    @property
    def ctype(self):
        return _CTYPES[self.data.dtype.name]

    def __call__(self, access):
        return Arg(self, None, None, access)


_CONSTS = {}


class Const(object):
    def __init__(self, dim, data, name, dtype=None):
        self.dim = tuple(np.atleast_1d(dim).astype(int).tolist())
        self.cdim = int(np.prod(self.dim))
        self.data = np.ascontiguousarray(np.array(data, dtype=dtype).reshape(self.dim))
        self.name = name
        _CONSTS[name] = self

    @property
    def ctype(self):
        return _CTYPES[self.data.dtype.name]

    def remove_from_namespace(self):
        _CONSTS.pop(self.name, None)


class Kernel(object):
    def __init__(self, code, name):
        self.code, self.name = code, name


class Sparsity(object):
    """CSR pattern from map pairs, built by the restated
    build_sparsity_pattern_seq (oracle_core.c), or by the reference's own
    compiled function when ``use_reference=True`` and it is available."""

    def __init__(self, maps, name=None, use_reference=False):
        if isinstance(maps, Map):
            maps = (maps, maps)
        if isinstance(maps[0], Map):
            maps = (maps,)
        self.maps = [tuple(p) for p in maps]
        self.rmaps = [p[0] for p in self.maps]
        self.cmaps = [p[1] for p in self.maps]
        self.nrows = self.rmaps[0].dataset.size
        self.ncols = self.cmaps[0].dataset.size
        self.dims = (self.rmaps[0].dataset.cdim, self.cmaps[0].dataset.cdim)
        if use_reference:
            from .reference import build_sparsity_reference
            self.rowptr, self.colidx, self.nnz = build_sparsity_reference(
                self.dims[0], self.dims[1], self.nrows, self.maps)
        else:
            self.rowptr, self.colidx, self.nnz = build_sparsity(self.dims[0], self.dims[1],
                                                                self.nrows, self.maps)
        self.nz = int(self.rowptr[-1])


def build_sparsity(rmult, cmult, nrows, maps):
    n = len(maps)
    keep = [np.ascontiguousarray(m.values, dtype=np.int32) for p in maps for m in p]
    rm = (C.c_void_p * n)(*[keep[2 * k].ctypes.data for k in range(n)])
    cm = (C.c_void_p * n)(*[keep[2 * k + 1].ctypes.data for k in range(n)])
    rd = (C.c_int * n)(*[p[0].dim for p in maps])
    cd = (C.c_int * n)(*[p[1].dim for p in maps])
    fs = (C.c_int * n)(*[p[0].iterset.size for p in maps])
    nnz, rowptr, colidx = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_int)()
    nz = C.c_int64()
    lib = core()
    rc = lib.oracle_build_sparsity(rmult, cmult, nrows, n, rm, rd, cm, cd, fs, C.byref(nnz),
                                   C.byref(rowptr), C.byref(colidx), C.byref(nz))
    if rc:
        raise ValueError("row map value outside the row set")
    lsize = nrows * rmult
    out = (np.ctypeslib.as_array(rowptr, (lsize + 1,)).copy(),
           np.ctypeslib.as_array(colidx, (max(nz.value, 1),))[:nz.value].copy(),
           np.ctypeslib.as_array(nnz, (max(lsize, 1),))[:lsize].copy())
    for p in (nnz, rowptr, colidx):
        lib.oracle_free(C.cast(p, C.c_void_p))
    return out


class Mat(object):
    def __init__(self, sparsity, dtype=np.float64, name=None):
        self.sparsity = sparsity
        self.dims = sparsity.dims
        self.array = np.zeros(sparsity.nz, dtype=np.float64)
        self.name = name

    @property
    def ctype(self):
        return "double"

    def __call__(self, path, access):
        rows, cols = path
        return Arg(self, (rows.map, cols.map), (rows.idx, cols.idx), access)

    @property
    def values(self):
        rp, ci = self.sparsity.rowptr, self.sparsity.colidx
        nr = self.sparsity.nrows * self.dims[0]
        nc = self.sparsity.ncols * self.dims[1]
        out = np.zeros((nr, nc))
        for r in range(nr):
            out[r, ci[rp[r]:rp[r + 1]]] = self.array[rp[r]:rp[r + 1]]
        return out

    def zero(self):
        self.array[:] = 0.0

    def zero_rows(self, rows, diag):
        rp, ci = self.sparsity.rowptr, self.sparsity.colidx
        for r in rows:
            seg = slice(rp[r], rp[r + 1])
            self.array[seg] = 0.0
            self.array[seg][ci[seg] == r] = diag


# --------------------------------------------------------------- codegen
def _kind(a):
    if isinstance(a.data, Global):
        return "gbl"
    if isinstance(a.data, Mat):
        return "mat"
    if a.map is IdentityMap:
        return "direct"
    if a.idx is None:
        return "vec"
    if isinstance(a.idx, IterationIndex):
        return "its"
    return "ind"


def _generate(kernel, extents, args, consts, openmp):
    """C source of the wrapper (sequential.py:55-72, host.py:91-322)."""
    decl, vec, zero, kargs, vaddto, saddto, ltens = [], [], [], [], [], [], []
    red_decl, red_init, red_fin = [], [], []
    p = 0
    for n, a in enumerate(args):
        k = _kind(a)
        t = a.data.ctype
        if k == "mat":
            decl.append("double *a%d = (double *)args[%d];" % (n, p))
            decl.append("const int *a%d_rp = (const int *)args[%d];" % (n, p + 1))
            decl.append("const int *a%d_ci = (const int *)args[%d];" % (n, p + 2))
            decl.append("const int *a%d_map = (const int *)args[%d];" % (n, p + 3))
            decl.append("const int *a%d_map2 = (const int *)args[%d];" % (n, p + 4))
            p += 5
        else:
            decl.append("%s *a%d = (%s *)args[%d];" % (t, n, t, p))
            p += 1
            if k in ("ind", "vec", "its"):
                decl.append("const int *a%d_map = (const int *)args[%d];" % (n, p))
                p += 1
        if k == "gbl":
            if a.access is READ:
                kargs.append("a%d" % n)
            elif not openmp:
                kargs.append("a%d" % n)
            else:
                red_decl.append("%s a%d_l[64][%d];" % (t, n, a.data.cdim))
                init = "(%s)0" % t if a.access is INC else "a%d[i]" % n
                red_init.append("for (int i = 0; i < %d; i++) a%d_l[tid][i] = %s;" % (a.data.cdim, n, init))
                if a.access is INC:
                    comb = "a%d[i] += a%d_l[th][i]" % (n, n)
                elif a.access is MIN:
                    comb = "a%d[i] = a%d[i] < a%d_l[th][i] ? a%d[i] : a%d_l[th][i]" % (n, n, n, n, n)
                else:
                    comb = "a%d[i] = a%d[i] > a%d_l[th][i] ? a%d[i] : a%d_l[th][i]" % (n, n, n, n, n)
                red_fin.append("for (int th = 0; th < nthread; th++) for (int i = 0; i < %d; i++) %s;"
                               % (a.data.cdim, comb))
                kargs.append("a%d_l[tid]" % n)
        elif k == "direct":
            kargs.append("a%d + (long long)i * %d" % (n, a.data.cdim))
        elif k == "ind":
            kargs.append("a%d + (long long)a%d_map[(long long)i * %d + %d] * %d" % (n, n, a.map.dim, a.idx, a.data.cdim))
        elif k == "its":
            kargs.append("a%d + (long long)a%d_map[(long long)i * %d + i_%d] * %d" % (n, n, a.map.dim, a.idx.index, a.data.cdim))
        elif k == "vec":
            ltens.append("%s *a%d_vec[%d];" % (t, n, a.map.dim))
            for r in range(a.map.dim):
                vec.append("a%d_vec[%d] = a%d + (long long)a%d_map[(long long)i * %d + %d] * %d;"
                           % (n, r, n, n, a.map.dim, r, a.data.cdim))
            kargs.append("a%d_vec" % n)
        elif k == "mat":
            rm, cm = a.data.dims
            rmap, cmap = a.map
            ins = 1 if a.access is WRITE else 0
            if rm * cm == 1:
                ltens.append("double p%d[%d][%d];" % (n, extents[0], extents[1]))
                zero.append("p%d[i_0][i_1] = 0.0;" % n)
                kargs.append("(double (*)[1])&p%d[i_0][i_1]" % n)
                saddto.append("err |= oracle_csr_addto_block(a%d, a%d_rp, a%d_ci, &p%d[0][0], %d, "
                              "a%d_map + (long long)i * %d, %d, a%d_map2 + (long long)i * %d, %d);"
                              % (n, n, n, n, rmap.dim, n, rmap.dim, cmap.dim, n, cmap.dim, ins))
            else:
                ltens.append("double p%d[%d][%d];" % (n, rm, cm))
                zero.append("memset(p%d, 0, sizeof(double) * %d);" % (n, rm * cm))
                kargs.append("p%d" % n)
                for r in range(rm):
                    for c in range(cm):
                        vaddto.append(
                            "err |= oracle_csr_addto_scalar(a%d, a%d_rp, a%d_ci, p%d[%d][%d], "
                            "%d * a%d_map[(long long)i * %d + i_0] + %d, %d * a%d_map2[(long long)i * %d + i_1] + %d, %d);"
                            % (n, n, n, n, r, c, rm, n, rmap.dim, r, cm, n, cmap.dim, c, ins))
    itargs = ["i_%d" % d for d in range(len(extents))]
    loops_open = "".join("for (int i_%d = 0; i_%d < %d; ++i_%d) {" % (d, d, e, d)
                         for d, e in enumerate(extents))
    loops_close = "}" * len(extents)
    const_decl = []
    const_init = []
    for c in consts:
        if c.cdim == 1:
            const_decl.append("static %s %s;" % (c.ctype, c.name))
        else:
            const_decl.append("static %s %s[%d];" % (c.ctype, c.name, c.cdim))
        const_init.append("memcpy(%s%s, consts[%d], sizeof(%s) * %d);" %
                          ("&" if c.cdim == 1 else "", c.name, len(const_init), c.ctype, c.cdim))
    body = """
{vecs}
{lo}
  {zero}
  {kname}({kargs});
  {vaddto}
{lc}
{saddto}
""".format(vecs="\n".join(vec), lo=loops_open, zero="\n".join(zero), kname=kernel.name,
           kargs=", ".join(kargs + itargs), vaddto="\n".join(vaddto), lc=loops_close,
           saddto="\n".join(saddto))
    src = ["#include <math.h>", "#include <string.h>", "#include <stdint.h>",
           "#ifdef _OPENMP", "#include <omp.h>", "#endif",
           "int oracle_csr_addto_scalar(double*, const int*, const int*, double, int, int, int);",
           "int oracle_csr_addto_block(double*, const int*, const int*, const double*, int, const int*, int, const int*, int);"]
    src += const_decl
    src += ["#define OP2_STRIDE(a, idx) a[idx]", _static_inline(kernel.code, kernel.name), "#undef OP2_STRIDE"]
    if not openmp:
        src.append("""
int wrap(int start, int end, void **args, void **consts) {
  int err = 0;
  %s
  %s
  %s
  for (int i = start; i < end; i++) {
  %s
  }
  return err;
}""" % ("\n  ".join(decl), "\n  ".join(ltens), "\n  ".join(const_init), body))
    else:
        src.append("""
int wrap(int part_size, int ncolors, const int *blkmap, const int *ncolblk, const int *nelems,
         void **args, void **consts) {
  int err = 0;
  %s
  %s
  int nthread = 1;
#ifdef _OPENMP
  nthread = omp_get_max_threads();
  if (nthread > 64) nthread = 64;
#endif
  %s
#pragma omp parallel num_threads(nthread)
  {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    %s
  }
  int boffset = 0;
  for (int col = 0; col < ncolors; col++) {
    int nblocks = ncolblk[col];
#pragma omp parallel num_threads(nthread) reduction(|:err)
    {
      int tid = 0;
#ifdef _OPENMP
      tid = omp_get_thread_num();
#endif
      %s
#pragma omp for schedule(static)
      for (int b = boffset; b < boffset + nblocks; b++) {
        int bid = blkmap[b];
        int first = bid * part_size;
        for (int i = first; i < first + nelems[bid]; i++) {
        %s
        }
      }
    }
    boffset += nblocks;
  }
  %s
  return err;
}""" % ("\n  ".join(decl), "\n  ".join(const_init), "\n  ".join(red_decl),
       "\n    ".join(red_init), "\n      ".join(ltens), body, "\n  ".join(red_fin)))
    return "\n".join(src)


def _static_inline(code, name):
    """The kernel code with its entry function made `static inline` (the
    reference compiled it `inline`, pyop2/host.py:230-239)."""
    import re
    m = re.search(r"(^|[;}\s])(void\s+%s\s*\()" % re.escape(name), code)
    if not m:
        return code
    return code[:m.start(2)] + "static inline " + code[m.start(2):]


_MODCACHE = {}
_CACHE_DIR = os.path.join(tempfile.gettempdir(), "op2b-oracle-%d" % os.getuid())


def _compile(src, openmp):
    key = hashlib.sha256((src + str(openmp)).encode()).hexdigest()
    if key in _MODCACHE:
        return _MODCACHE[key]
    os.makedirs(_CACHE_DIR, exist_ok=True)
    so = os.path.join(_CACHE_DIR, key + ".so")
    if not os.path.exists(so):
        cfile = os.path.join(_CACHE_DIR, key + ".c")
        with open(cfile, "w") as f:
            f.write(src)
        cmd = ["gcc", "-O2", "-std=gnu99", "-shared", "-fPIC", cfile, "-o", so + ".tmp%d" % os.getpid(),
               _build.build_oracle(), "-lm", "-Wl,-rpath," + os.path.dirname(_build.build_oracle())]
        if openmp:
            cmd.insert(1, "-fopenmp")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError("oracle compile failed:\n%s\n%s" % (r.stderr, src))
        os.replace(so + ".tmp%d" % os.getpid(), so)
    core()
    lib = C.CDLL(so)
    lib.wrap.restype = C.c_int
    _MODCACHE[key] = lib
    return lib


def _marshal(args):
    ptrs, keep = [], []
    for a in args:
        k = _kind(a)
        if k == "mat":
            sp = a.data.sparsity
            for arr in (a.data.array, sp.rowptr, sp.colidx, a.map[0].values, a.map[1].values):
                keep.append(arr)
                ptrs.append(arr.ctypes.data)
        else:
            keep.append(a.data.data)
            ptrs.append(a.data.data.ctypes.data)
            if k in ("ind", "vec", "its"):
                keep.append(a.map.values)
                ptrs.append(a.map.values.ctypes.data)
    return (C.c_void_p * max(len(ptrs), 1))(*ptrs), keep


def par_loop(kernel, itspace, *args, openmp=False, part_size=1024, timer=None, span=None):
    """Run the loop with sequential (or restated OpenMP) semantics.
    ``timer``, if given, is called with the wall seconds of the element loop
    alone (code generation, compilation and planning excluded).  ``span`` =
    (start, end) runs elements [start, end) only, as the sequential backend's
    wrapper does for the core / owned / execute-halo ranges of a
    partitioned set (sequential.py:96-117; sequential only)."""
    import time
    if isinstance(itspace, Set):
        itspace = IterationSpace(itspace, ())
    consts = sorted(_CONSTS.values(), key=lambda c: c.name)
    src = _generate(kernel, itspace.extents, args, consts, openmp)
    lib = _compile(src, openmp)
    cargs, keep = _marshal(args)
    cvals = [np.ascontiguousarray(c.data) for c in consts]
    cptr = (C.c_void_p * max(len(cvals), 1))(*[c.ctypes.data for c in cvals])
    n = itspace.iterset.size
    start, end = (0, n) if span is None else (int(span[0]), int(span[1]))
    if not 0 <= start <= end <= n or (openmp and span is not None):
        raise ValueError("span %s of a set of %d elements" % (span, n))
    if not openmp:
        t0 = time.perf_counter()
        err = lib.wrap(start, end, cargs, cptr)
        dt = time.perf_counter() - t0
    else:
        from .plan import plan as make_plan
        need = any(_kind(a) in ("ind", "vec", "its", "mat") for a in args)
        if need:
            pl = make_plan(itspace.iterset, _unwind(itspace, args), partition_size=part_size,
                           matrix_coloring=True, staging=False, thread_coloring=False)
            ncolors, blkmap, ncolblk, nelems = pl.ncolors, pl.blkmap, pl.ncolblk, pl.nelems
        else:
            nb = (n + part_size - 1) // part_size
            ncolors, blkmap = 1, np.arange(nb, dtype=np.int32)
            ncolblk = np.array([nb], np.int32)
            nelems = np.array([min(part_size, n - b * part_size) for b in range(nb)], np.int32)
        blkmap = np.ascontiguousarray(blkmap, np.int32)
        ncolblk = np.ascontiguousarray(ncolblk, np.int32)
        nelems = np.ascontiguousarray(nelems, np.int32)
        t0 = time.perf_counter()
        err = lib.wrap(part_size, ncolors, blkmap.ctypes.data_as(C.c_void_p),
                       ncolblk.ctypes.data_as(C.c_void_p), nelems.ctypes.data_as(C.c_void_p),
                       cargs, cptr)
        dt = time.perf_counter() - t0
    if timer is not None:
        timer(dt)
    if err:
        raise ValueError("Mat insertion outside the Sparsity pattern")


def _unwind(itspace, args):
    """Unwind vec-map and itspace args (pyop2/device.py:390-419)."""
    out = []
    for a in args:
        k = _kind(a)
        if k == "vec":
            out += [Arg(a.data, a.map, r, a.access) for r in range(a.map.dim)]
        elif k == "its":
            out += [Arg(a.data, a.map, r, a.access) for r in range(itspace.extents[a.idx.index])]
        else:
            out.append(a)
    return out
