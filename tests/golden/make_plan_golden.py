"""Generate tests/golden/plan_reference.npz: plans built by the reference's
own Plan class (pyop2/plan.pyx, translated by Cython and compiled by
oracle/build.py; run through oracle/reference.py) for a set of seeded loops.

Run in a container that has the reference sources (found where
oracle/build.py looks for them); the output is committed so tests never need
the reference at run time.  Each case stores its loop description (Map values, Dat sizes,
the unwound arguments) and every array and scalar the reference Plan holds
(partition, staging, thread and block colouring).
"""

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from conftest import py2_shuffle, reference_seed  # noqa: E402
from oracle import reference  # noqa: E402
from pyop2_b200.workloads import meshes  # noqa: E402


def cases():
    """(name, case, partition_size, matrix_coloring) of every fixture."""
    out = []
    rng = np.random.default_rng(2024)
    m = rng.integers(0, 300, size=(1000, 2)).astype(np.int32)
    m[::17, 1] = m[::17, 0]                      # an element touching one target twice
    for ps in (64, 128):
        out.append(("random_edges_ps%d" % ps, reference.plan_case(
            1000, {"m": (m, 300)},
            {"x": (300, "float64", 2), "y": (300, "float64", 1), "w": (1000, "float64", 1)},
            [("x", "m", 0, "INC"), ("x", "m", 1, "INC"), ("y", "m", 0, "READ"), ("y", "m", 1, "READ"),
             ("w", None, None, "READ")]), ps, False))
    g = meshes.airfoil_grid(20, 10, 3)
    pedge = np.asarray(g.pedge, np.int32).reshape(-1, 2)
    pecell = np.asarray(g.pecell, np.int32).reshape(-1, 2)
    out.append(("airfoil_res_calc_20x10", reference.plan_case(
        g.nedges, {"pedge": (pedge, g.nnodes), "pecell": (pecell, g.ncells)},
        {"x": (g.nnodes, "float64", 2), "q": (g.ncells, "float64", 4), "adt": (g.ncells, "float64", 1),
         "res": (g.ncells, "float64", 4)},
        [("x", "pedge", 0, "READ"), ("x", "pedge", 1, "READ"), ("q", "pecell", 0, "READ"),
         ("q", "pecell", 1, "READ"), ("adt", "pecell", 0, "READ"), ("adt", "pecell", 1, "READ"),
         ("res", "pecell", 0, "INC"), ("res", "pecell", 1, "INC")]), 64, False))
    coords, elem = meshes.square_p1(6)
    elem = np.asarray(elem, np.int32)
    nn = coords.shape[0]
    p1 = reference.plan_case(
        elem.shape[0], {"en": (elem, nn), "evn": (elem.copy(), nn)},
        {"coords": (nn, "float64", 2), "b": (nn, "float64", 1)},
        [("A", "en", None, "INC"), ("coords", "evn", 0, "READ"), ("coords", "evn", 1, "READ"),
         ("coords", "evn", 2, "READ")], mats={"A": "en"})
    out.append(("p1_mass_matrix_coloring", p1, 16, True))
    out.append(("p1_mass_no_matrix_coloring", p1, 16, False))
    rhs = reference.plan_case(
        elem.shape[0], {"en": (elem, nn), "evn": (elem.copy(), nn)},
        {"coords": (nn, "float64", 2), "b": (nn, "float64", 1)},
        [("b", "en", 0, "INC"), ("b", "en", 1, "INC"), ("b", "en", 2, "INC"),
         ("coords", "evn", 0, "READ"), ("coords", "evn", 1, "READ"), ("coords", "evn", 2, "READ")])
    out.append(("p1_rhs_ps32", rhs, 32, False))
    one = np.zeros((150, 1), np.int32)           # every element adds to target 0
    out.append(("one_target_ps80", reference.plan_case(
        150, {"m0": (one, 4)}, {"z": (4, "int32", 1)}, [("z", "m0", 0, "INC")]), 80, False))
    m1 = rng.integers(0, 50, size=(400, 1)).astype(np.int32)
    m2 = rng.integers(0, 50, size=(400, 2)).astype(np.int32)
    out.append(("one_dat_two_maps", reference.plan_case(
        400, {"m1": (m1, 50), "m2": (m2, 50)}, {"v": (50, "float32", 3)},
        [("v", "m1", 0, "INC"), ("v", "m2", 0, "INC"), ("v", "m2", 1, "INC")]), 40, False))
    # the loops of test/unit/test_plan.py: a shuffled one-to-one map written
    # (:73-83, partition 128), a chain of 4095 edges reading both ends (:85-109,
    # partition 96) and the two-element RHS (:111-142, partition 2)
    n = 4096
    u = np.arange(n, dtype=np.int32)
    py2_shuffle(u, reference_seed)
    out.append(("test_plan_onecolor_wo", reference.plan_case(
        n, {"u": (u.reshape(n, 1), n)}, {"x": (n, "uint32", 1)}, [("x", "u", 0, "WRITE")]), 128, False))
    e = np.array([(i, i + 1) for i in range(n - 1)], dtype=np.int32)
    out.append(("test_plan_2d_map", reference.plan_case(
        n - 1, {"e2n": (e, n)}, {"node_vals": (n, "uint32", 1), "edge_vals": (n - 1, "uint32", 1)},
        [("node_vals", "e2n", 0, "READ"), ("node_vals", "e2n", 1, "READ"),
         ("edge_vals", None, None, "WRITE")]), 96, False))
    en = np.array([0, 1, 3, 2, 3, 1], dtype=np.int32).reshape(2, 3)
    out.append(("test_plan_rhs", reference.plan_case(
        2, {"elem_node": (en, 4)},
        {"b": (4, "float64", 1), "coords": (4, "float64", 2), "f": (4, "float64", 1)},
        [("b", "elem_node", 0, "INC"), ("b", "elem_node", 1, "INC"), ("b", "elem_node", 2, "INC"),
         ("coords", "elem_node", 0, "READ"), ("coords", "elem_node", 1, "READ"),
         ("coords", "elem_node", 2, "READ"), ("f", "elem_node", 0, "READ"),
         ("f", "elem_node", 1, "READ"), ("f", "elem_node", 2, "READ")]), 2, False))
    return out


def main():
    store, index = {}, []
    for name, case, ps, mc in cases():
        r = reference.plan_reference(case, ps, matrix_coloring=mc)
        meta = {"name": name, "size": case["size"], "partition_size": ps, "matrix_coloring": mc,
                "maps": {k: int(t) for k, (v, t) in case["maps"].items()},
                "dats": {k: [int(s), str(np.dtype(d)), int(c)] for k, (s, d, c) in case["dats"].items()},
                "mats": case["mats"], "args": case["args"],
                "scalars": {f: int(r[f]) for f in ("nblocks", "nshared", "ncolors")}}
        index.append(meta)
        for k, (v, t) in case["maps"].items():
            store["%s/map/%s" % (name, k)] = np.asarray(v, np.int32)
        for f in reference.PLAN_FIELDS:
            if f not in meta["scalars"]:
                store["%s/%s" % (name, f)] = np.asarray(r[f])
    store["index"] = np.frombuffer(json.dumps(index).encode(), dtype=np.uint8)
    path = os.path.join(HERE, "plan_reference.npz")
    np.savez_compressed(path, **store)
    print(path, os.path.getsize(path), "bytes,", len(index), "cases")


if __name__ == "__main__":
    main()
