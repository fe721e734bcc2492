"""Owner-computes partitioning of a mesh across ranks.

The reference leaves partitioning to the caller: a rank declares its Sets
with four sizes -- core, owned, execute halo, non-execute halo
(pyop2/base.py:261-357) -- its Maps in that local numbering, and a
:class:`Halo` per Set naming the owned elements it sends to each peer and
the halo elements it receives from each (pyop2/base.py:402-505;
demo/mass2d_mpi.py writes them by hand).  This module derives all of it from
a global mesh and an owner rank per element, with the reference's
definitions:

* owned: the elements the rank owns;
* execute halo (sets iterated through Maps): elements owned elsewhere that
  reach an element owned here through one of the set's Maps -- loops that
  increment through a Map run them too, so contributions to owned rows are
  complete without a reverse exchange (pyop2/sequential.py:113-116);
* non-execute halo: elements owned elsewhere that the owned or execute-halo
  elements of some set reach through a Map (read, never executed);
* core: owned elements whose every Map target is owned here, so a loop can
  run them before the halo exchange completes (pyop2/sequential.py:96-103).

Local numbering per set: core, the other owned elements, execute halo,
non-execute halo, each in increasing global id.  A halo's sends to rank q
and q's receives from this rank list the same elements in increasing global
id, so the two sides pair up row by row.

Pure host code (numpy); the result feeds ``op2.Set`` / ``op2.Map`` /
``op2.Halo`` / ``op2.Dat`` of each rank.
"""

import numpy as np


class LocalSet(object):
    """One set on one rank: ``sizes`` (core, owned, exec, total), ``l2g``
    (global id of each local element), ``sends`` / ``receives`` (per peer
    rank, local ids)."""

    def __init__(self, name, sizes, l2g):
        self.name = name
        self.sizes = tuple(int(s) for s in sizes)
        self.l2g = l2g
        self.sends = None
        self.receives = None

    def g2l(self, nglobal):
        """Global id -> local id (-1 where the element is not on this rank)."""
        out = np.full(nglobal, -1, dtype=np.int64)
        out[self.l2g] = np.arange(self.l2g.size)
        return out

    def local_rows(self, values):
        """Rows of a global per-element array in this rank's local order."""
        return np.ascontiguousarray(np.asarray(values)[self.l2g])


class LocalMesh(object):
    """Everything rank ``rank`` declares: ``sets`` (name -> LocalSet) and
    ``maps`` (name -> (from set, to set, local values))."""

    def __init__(self, rank, nranks):
        self.rank, self.nranks = rank, nranks
        self.sets = {}
        self.maps = {}


def partition(sets, maps, owner, nranks):
    """Partition a global mesh.

    ``sets``: name -> global size; ``maps``: name -> (from set, to set,
    values [n_from][arity]); ``owner``: set name -> owner rank of every
    element.  Returns one :class:`LocalMesh` per rank."""
    sets = {k: int(v) for k, v in sets.items()}
    owner = {k: np.asarray(v, dtype=np.int64) for k, v in owner.items()}
    for k, n in sets.items():
        if owner[k].shape != (n,):
            raise ValueError("owner of set %s has shape %s, expected (%d,)" % (k, owner[k].shape, n))
        if n and (owner[k].min() < 0 or owner[k].max() >= nranks):
            raise ValueError("owner of set %s outside [0, %d)" % (k, nranks))
    vals = {}
    for name, (src, dst, v) in maps.items():
        v = np.asarray(v, dtype=np.int64).reshape(sets[src], -1)
        if v.size and (v.min() < 0 or v.max() >= sets[dst]):
            raise ValueError("map %s has values outside [0, %d)" % (name, sets[dst]))
        vals[name] = (src, dst, v)
    from_maps = {k: [m for m, (s, _, _) in vals.items() if s == k] for k in sets}

    meshes = []
    halo_of = []          # per rank: set name -> global ids of its halo (exec + non-exec)
    for r in range(nranks):
        mine = {k: owner[k] == r for k in sets}
        execm = {}
        for k in sets:
            reach = np.zeros(sets[k], dtype=bool)
            for m in from_maps[k]:
                _, dst, v = vals[m]
                reach |= mine[dst][v].any(axis=1)
            execm[k] = reach & ~mine[k]
        refd = {k: np.zeros(sets[k], dtype=bool) for k in sets}
        for m, (src, dst, v) in vals.items():
            rows = mine[src] | execm[src]
            refd[dst][v[rows].ravel()] = True
        local = LocalMesh(r, nranks)
        halos = {}
        for k in sets:
            core = mine[k].copy()
            for m in from_maps[k]:
                _, dst, v = vals[m]
                core &= mine[dst][v].all(axis=1)
            owned_rest = mine[k] & ~core
            nonexec = refd[k] & ~mine[k] & ~execm[k]
            parts = [np.flatnonzero(core), np.flatnonzero(owned_rest), np.flatnonzero(execm[k]),
                     np.flatnonzero(nonexec)]
            l2g = np.concatenate(parts).astype(np.int64)
            c = np.cumsum([p.size for p in parts])
            local.sets[k] = LocalSet(k, c, l2g)
            halos[k] = l2g[c[1]:]
        meshes.append(local)
        halo_of.append(halos)

    for r, local in enumerate(meshes):
        g2l = {k: s.g2l(sets[k]) for k, s in local.sets.items()}
        for k, s in local.sets.items():
            # both sides in increasing global id (the halo's local ids grow
            # with global id only inside its exec and non-exec parts)
            halo = halo_of[r][k]
            none = np.zeros(0, np.int32)
            s.receives = [g2l[k][np.sort(halo[owner[k][halo] == q])].astype(np.int32)
                          if q != r else none for q in range(nranks)]
            s.sends = [g2l[k][np.sort(halo_of[q][k][owner[k][halo_of[q][k]] == r])].astype(np.int32)
                       if q != r else none for q in range(nranks)]
        for m, (src, dst, v) in vals.items():
            s = local.sets[src]
            lv = g2l[dst][v[s.l2g]]
            # rows of non-execute halo elements may reach targets this rank does
            # not hold; they are never executed
            lv[lv < 0] = 0
            local.maps[m] = (src, dst, lv.astype(np.int32))
    return meshes
