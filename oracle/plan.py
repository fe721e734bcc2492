"""CPU oracle: plan.pyx restated.  TEST INFRASTRUCTURE ONLY.

``plan(iterset, args, partition_size, matrix_coloring, staging,
thread_coloring)`` returns the arrays Plan.__cinit__ builds
(pyop2/plan.pyx:93-376):

* partition (:107-110): ``nblocks``, ``nelems``, ``offset``;
* staging (:112-212), restated with numpy.unique exactly as the reference
  does: ``ind_map`` (per (Dat, Map) pair, blocks' sorted unique values, padded
  with -1 to nidx*size), ``loc_map`` (int16), ``ind_sizes``, ``ind_offs``,
  ``nindirect``, ``nshared``;
* colouring (:214-376) by oracle_core.c's oracle_plan_color (same loops):
  ``thrcol``, ``nthrcol``, ``ncolors``, ``ncolblk``, ``blkmap``.

``args`` are unwound oracle Args (Dat args with an int idx, Mat args).
Note: the reference stores the inverse of column ``ii[i]`` under index
``sorted(ii)[i]`` (:151-152), which only matches for ascending indices; this
restatement indexes by the actual index, which equals the reference whenever
the indices of a pair are listed in ascending order (every reference use).
"""

import ctypes as C
import math

import numpy as np

from .seq import Mat, core


def _align(n, a=16):
    return ((n + a - 1) // a) * a


class OraclePlan(object):
    pass


def plan(iset, args, partition_size=1, matrix_coloring=False, staging=True, thread_coloring=True):
    ps = int(partition_size)
    P = OraclePlan()
    size = iset.size
    P.nblocks = int(math.ceil(size / float(ps)))
    P.nelems = np.array([min(ps, size - b * ps) for b in range(P.nblocks)], dtype=np.int32)
    P.offset = np.array([b * ps for b in range(P.nblocks)], dtype=np.int32)
    dargs = [a for a in args if not isinstance(a.data, Mat)]
    if staging:
        d = []
        for a in dargs:
            if a.map is not None and a.idx is not None and not any(a.data is x[0] and a.map is x[1] for x in d):
                d.append((a.data, a.map))

        def indices(dat, m):
            return [a.idx for a in dargs if a.data is dat and a.map is m]

        inds, locs, sizes = {}, {}, {}
        for pi in range(P.nblocks):
            start = pi * ps
            end = start + P.nelems[pi]
            for k, (dat, m) in enumerate(d):
                ii = indices(dat, m)
                u, inv = np.unique(m.values[start:end][:, ii], return_inverse=True)
                inv = inv.reshape(-1)
                inds[(k, pi)] = u.astype(np.int32)
                sizes[(k, pi)] = len(u)
                for j, ix in enumerate(ii):
                    locs[(k, ix, pi)] = inv[j::len(ii)]
        parts = []
        for k, (dat, m) in enumerate(d):
            cum = 0
            for pi in range(P.nblocks):
                parts.append(inds[(k, pi)])
                cum += sizes[(k, pi)]
            parts.append(np.full(len(indices(dat, m)) * size - cum, -1, dtype=np.int32))
        P.ind_map = np.concatenate(parts) if parts else np.zeros(0, np.int32)
        P.ind_sizes = np.array([sizes[(k, pi)] for pi in range(P.nblocks) for k in range(len(d))],
                               dtype=np.int32)
        P.nindirect = np.array([sum(sizes[(k, pi)] for pi in range(P.nblocks)) for k in range(len(d))],
                               dtype=np.int32)
        lp = []
        for k, (dat, m) in enumerate(d):
            for ix in indices(dat, m):
                for pi in range(P.nblocks):
                    lp.append(locs[(k, ix, pi)].astype(np.int16))
        P.loc_map = np.concatenate(lp) if lp else np.zeros(0, np.int16)
        offs, run = [], [0] * len(d)
        for pi in range(P.nblocks):
            for k in range(len(d)):
                offs.append(run[k])
                run[k] += sizes[(k, pi)]
        P.ind_offs = np.array(offs, dtype=np.int32)
        P.nshared = max([sum(_align(sizes[(k, pi)] * dat.data.dtype.itemsize * dat.cdim)
                             for k, (dat, m) in enumerate(d)) for pi in range(P.nblocks)] or [0])
        P.ninds = len(d)
    # colouring
    race = []
    for a in args:
        if not isinstance(a.data, Mat) and a.map is not None and a.access._mode == "INC" and a.idx is not None:
            g = next((r for r in race if r[0] is a.data), None)
            if g is None:
                g = [a.data, a.data.dataset.size, []]
                race.append(g)
            g[2].append((a.map, a.idx))
        elif matrix_coloring and isinstance(a.data, Mat):
            g = next((r for r in race if r[0] is a.data), None)
            rmap = a.map[0]
            if g is None:
                g = [a.data, rmap.dataset.size, []]
                race.append(g)
            g[2] += [(rmap, r) for r in range(rmap.dim)]
    nrace = len(race)
    ents = [e for g in race for e in g[2]]
    keep = [np.ascontiguousarray(m.values, np.int32) for m, _ in ents]
    maps = (C.c_void_p * max(len(ents), 1))(*[k.ctypes.data for k in keep])
    dims = (C.c_int * max(len(ents), 1))(*[m.dim for m, _ in ents])
    idxs = (C.c_int * max(len(ents), 1))(*[ix for _, ix in ents])
    rsize = (C.c_int * max(nrace, 1))(*[g[1] for g in race])
    rcount = (C.c_int * max(nrace, 1))(*[len(g[2]) for g in race])
    thrcol = np.empty(size, np.int32)
    nthrcol = np.zeros(P.nblocks, np.int32)
    pcol = np.empty(P.nblocks, np.int32)
    nel = np.ascontiguousarray(P.nelems)
    core().oracle_plan_color(P.nblocks, nel.ctypes.data_as(C.c_void_p), nrace, rsize, rcount, maps,
                             dims, idxs, int(bool(thread_coloring)), thrcol.ctypes.data_as(C.c_void_p),
                             nthrcol.ctypes.data_as(C.c_void_p), pcol.ctypes.data_as(C.c_void_p))
    P.thrcol = thrcol
    P.nthrcol = nthrcol
    P.pcolors = pcol
    P.ncolors = int(pcol.max()) + 1 if P.nblocks else 0
    P.ncolblk = np.bincount(pcol).astype(np.int32) if P.nblocks else np.zeros(0, np.int32)
    P.blkmap = np.argsort(pcol, kind='mergesort').astype(np.int32)
    return P
