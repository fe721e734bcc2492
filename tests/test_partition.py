"""The owner-computes partitioner (pyop2_b200/partition.py) on the airfoil
mesh: the set sizes, halos and local Maps a distributed run declares
(pyop2/base.py:261-357 for the four sizes, :402-505 for Halos) satisfy the
reference's definitions.  Host only."""

import numpy as np
import pytest

from pyop2_b200 import partition as P
from pyop2_b200.workloads import airfoil, meshes

_MAPS = {"pedge": ("edges", "nodes"), "pecell": ("edges", "cells"), "pbedge": ("bedges", "nodes"),
         "pbecell": ("bedges", "cells"), "pcell": ("cells", "nodes")}


def _global_maps(g):
    return {"pedge": np.asarray(g.pedge).reshape(-1, 2), "pecell": np.asarray(g.pecell).reshape(-1, 2),
            "pbedge": np.asarray(g.pbedge).reshape(-1, 2),
            "pbecell": np.asarray(g.pbecell).reshape(-1, 1),
            "pcell": np.asarray(g.pcell).reshape(-1, 4)}


@pytest.mark.parametrize("nranks", [1, 2, 3])
def test_airfoil_partition_invariants(nranks):
    g = meshes.airfoil_grid(24, 12, 1)
    parts = airfoil.partition_grid(g, nranks)
    gm = _global_maps(g)
    sizes = {"nodes": g.nnodes, "edges": g.nedges, "bedges": g.nbedges, "cells": g.ncells}
    # owned elements of every set: disjoint across ranks and covering the set
    for k, n in sizes.items():
        owned = np.concatenate([p.sets[k].l2g[:p.sets[k].sizes[1]] for p in parts])
        assert np.array_equal(np.sort(owned), np.arange(n)), k
    for r, p in enumerate(parts):
        for k, ls in p.sets.items():
            core, owned, ex, tot = ls.sizes
            assert 0 <= core <= owned <= ex <= tot == ls.l2g.size
            assert np.unique(ls.l2g).size == tot
        for m, (src, dst) in _MAPS.items():
            ls, lt = p.sets[src], p.sets[dst]
            local = p.maps[m][2]
            run = ls.sizes[2]                          # executed: owned + exec halo
            # executed elements reach local targets, the same ones as globally
            assert np.array_equal(lt.l2g[local[:run]], gm[m][ls.l2g[:run]]), m
            # core elements reach owned targets only
            assert (local[:ls.sizes[0]] < lt.sizes[1]).all(), m
        for k, ls in p.sets.items():
            reach_owned = np.zeros(ls.sizes[3], bool)
            reach_halo = np.zeros(ls.sizes[3], bool)
            for m, (src, dst) in _MAPS.items():
                if src == k:
                    lt = p.sets[dst]
                    reach_owned |= (p.maps[m][2] < lt.sizes[1]).any(axis=1)
                    reach_halo |= (p.maps[m][2] >= lt.sizes[1]).any(axis=1)
            # exec-halo elements reach an owned target; owned elements outside
            # the core reach a halo target
            assert reach_owned[ls.sizes[1]:ls.sizes[2]].all(), k
            assert reach_halo[ls.sizes[0]:ls.sizes[1]].all(), k
        # sends pair with the peers' receives, element by element
        for k, ls in p.sets.items():
            assert ls.sends[r].size == 0 and ls.receives[r].size == 0
            for q, peer in enumerate(parts):
                if q == r:
                    continue
                mine = ls.l2g[ls.sends[q]]
                theirs = peer.sets[k].l2g[peer.sets[k].receives[r]]
                assert np.array_equal(mine, theirs), (k, r, q)
                assert (ls.sends[q] < ls.sizes[1]).all()
                assert (peer.sets[k].receives[r] >= peer.sets[k].sizes[1]).all()
        # every halo element is received from its owner
        for k, ls in p.sets.items():
            got = np.sort(np.concatenate([ls.receives[q] for q in range(nranks)]))
            assert np.array_equal(got, np.arange(ls.sizes[1], ls.sizes[3])), k


def test_single_rank_is_the_whole_mesh():
    g = meshes.airfoil_grid(12, 6, 0)
    (p,) = airfoil.partition_grid(g, 1)
    for k, ls in p.sets.items():
        assert ls.sizes[1] == ls.sizes[2] == ls.sizes[3] == ls.l2g.size
    gm = _global_maps(g)
    for m, (src, dst) in _MAPS.items():
        assert np.array_equal(p.sets[dst].l2g[p.maps[m][2]], gm[m][p.sets[src].l2g])


def test_bad_input_is_rejected():
    with pytest.raises(ValueError):
        P.partition({"a": 3}, {}, {"a": np.array([0, 1, 2])}, 2)
    with pytest.raises(ValueError):
        P.partition({"a": 2, "b": 2}, {"m": ("a", "b", np.array([[0], [2]]))},
                    {"a": np.zeros(2, int), "b": np.zeros(2, int)}, 1)
