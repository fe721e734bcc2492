"""The plan restatement (oracle/plan.py with oracle/csrc/oracle_core.c)
against plans built by the reference's own Plan class (pyop2/plan.pyx,
compiled from the reference sources; fixtures in
tests/golden/plan_reference.npz made by tests/golden/make_plan_golden.py):
partition, staging arrays (ind_map, loc_map, ind_sizes, ind_offs,
nindirect, nshared), thread colours and block colours, equal field by field.
The device plan builder is checked against the same restatement on the GPU
(test_gpu_plan_sparsity.py), so these fixtures pin it too.  When the
compiled reference is present, seeded random loops are also compared live.
CPU only."""

import json
import os

import numpy as np
import pytest

from oracle import plan as oplan
from oracle import reference, seq

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "plan_reference.npz")
ACCESS = {"READ": seq.READ, "WRITE": seq.WRITE, "RW": seq.RW, "INC": seq.INC}


def _oracle_plan(size, maps, dats, mats, args, ps, mc):
    """The oracle plan of a loop given as plain data (the plan_case form)."""
    it = seq.Set(size, 1, "it")
    sets = {}

    def target(n):
        if n not in sets:
            sets[n] = seq.Set(n, 1)
        return sets[n]
    M = {k: seq.Map(it, target(t), np.asarray(v).shape[1], v, k) for k, (v, t) in maps.items()}
    D = {}
    for k, (s, dt, c) in dats.items():
        D[k] = seq.Dat(seq.Set(s, c), None, np.dtype(dt), k)
    for k, r in mats.items():
        D[k] = seq.Mat(seq.Sparsity((M[r], M[r])), np.float64, k)
    a = []
    for name, mname, idx, acc in args:
        if name in mats:
            a.append(D[name]((M[mname][seq.i[0]], M[mname][seq.i[1]]), ACCESS[acc]))
        elif mname is None:
            a.append(seq.Arg(D[name], None, None, ACCESS[acc]))
        else:
            a.append(D[name](M[mname][idx], ACCESS[acc]))
    return oplan.plan(it, a, partition_size=ps, matrix_coloring=mc)


def _compare(P, ref):
    for f in reference.PLAN_FIELDS:
        got = getattr(P, f)
        want = ref[f]
        if np.ndim(want) == 0:
            assert int(got) == int(want), f
        else:
            np.testing.assert_array_equal(np.asarray(got).ravel(), np.asarray(want).ravel(), err_msg=f)
            assert np.asarray(got).dtype == np.asarray(want).dtype or f == "loc_map" and want.size == 0, f


def _fixtures():
    z = np.load(GOLDEN)
    index = json.loads(bytes(z["index"]).decode())
    return z, index


_NCASES = len(_fixtures()[1])


@pytest.mark.parametrize("k", range(_NCASES))
def test_oracle_plan_equals_reference_fixture(k):
    z, index = _fixtures()
    c = index[k]
    n = c["name"]
    maps = {m: (z["%s/map/%s" % (n, m)], t) for m, t in c["maps"].items()}
    ref = {f: z["%s/%s" % (n, f)] for f in reference.PLAN_FIELDS if f not in c["scalars"]}
    ref.update(c["scalars"])
    P = _oracle_plan(c["size"], maps, {d: tuple(v) for d, v in c["dats"].items()}, c["mats"],
                     [tuple(a) for a in c["args"]], c["partition_size"], c["matrix_coloring"])
    _compare(P, ref)


@pytest.mark.skipif(not reference.plan_available(), reason="compiled reference plan.pyx absent")
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_oracle_plan_equals_live_reference(seed):
    rng = np.random.default_rng(seed)
    size, nt = int(rng.integers(50, 700)), int(rng.integers(5, 200))
    ar = int(rng.integers(1, 5))
    m = rng.integers(0, nt, size=(size, ar)).astype(np.int32)
    case = reference.plan_case(size, {"m": (m, nt)}, {"x": (nt, "float64", 3), "y": (nt, "int32", 1)},
                               [("x", "m", r, "INC") for r in range(ar)] +
                               [("y", "m", r, "READ") for r in range(ar)])
    ps = int(rng.choice([8, 32, 100, 256]))
    ref = reference.plan_reference(case, ps)
    P = _oracle_plan(size, case["maps"], case["dats"], {}, case["args"], ps, False)
    _compare(P, ref)
