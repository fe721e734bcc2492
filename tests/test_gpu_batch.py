"""Batched loops on the GPU: many instances of one loop signature in one
launch, checked against the same loops run one at a time through op2 and
against the oracle.

Tolerances: direct loops and Global reductions of a batch are compared bit
for bit with the batch of one (a segment's reduction order depends only on
its own size and the tile); INC through Maps (atomic adds) within 1e-12
normwise relative, as in the single-loop parity tests."""

import numpy as np
import pytest

from conftest import rel_err
from oracle import seq
from pyop2_b200.workloads import fem, meshes

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture
def op2(backend):
    from pyop2_b200 import op2 as _op2
    return _op2


def _direct_instances(op2, sizes, seed):
    from pyop2_b200 import batch
    rng = np.random.default_rng(seed)
    k = op2.Kernel("""
void scale_sum(double *x, double *y, double *s, double *mn, double *mx) {
  y[0] = 2.0 * x[0] + x[1];
  y[1] = x[0] * x[1];
  s[0] += y[0];
  s[1] += y[1] * y[1];
  if (x[0] < mn[0]) mn[0] = x[0];
  if (x[1] > mx[0]) mx[0] = x[1];
}""", "scale_sum")
    out = []
    for n in sizes:
        st = op2.Set(int(n), 2)
        x = op2.Dat(st, rng.standard_normal((int(n), 2)), np.float64)
        y = op2.Dat(st, np.zeros((int(n), 2)), np.float64)
        s = op2.Global(2, (0.0, 0.0), np.float64)
        mn = op2.Global(1, 1e300, np.float64)
        mx = op2.Global(1, -1e300, np.float64)
        args = (x(op2.IdentityMap, op2.READ), y(op2.IdentityMap, op2.WRITE), s(op2.INC),
                mn(op2.MIN), mx(op2.MAX))
        out.append(dict(k=k, set=st, x=x, y=y, s=s, mn=mn, mx=mx, args=args,
                        inst=batch.LoopInstance(k, st, *args)))
    return out


@pytest.mark.parametrize("bs,ept", [(128, 1), (256, 2), (512, 4)])
def test_direct_batch_matches_numpy_and_is_mix_independent(op2, bs, ept):
    from pyop2_b200 import batch
    sizes = [1, 0, 300, 4097, 77, 20000, 513]
    mix = _direct_instances(op2, sizes, 1)
    batch.BatchLoop([m["inst"] for m in mix], block_size=bs, elems_per_thread=ept).launch()
    for m in mix:
        x = m["x"].data_ro
        y = np.stack([2.0 * x[:, 0] + x[:, 1], x[:, 0] * x[:, 1]], axis=1) if len(x) else x
        np.testing.assert_array_equal(m["y"].data_ro, y)
        if len(x):
            assert rel_err(m["s"].data_ro, [y[:, 0].sum(), (y[:, 1] ** 2).sum()]) < TOL
            assert m["mn"].data_ro[0] == x[:, 0].min()
            assert m["mx"].data_ro[0] == x[:, 1].max()
        else:
            assert m["s"].data_ro.tolist() == [0.0, 0.0]
    # the same instance (same data) alone gives bit-identical Globals
    again = _direct_instances(op2, sizes, 1)
    batch.BatchLoop([again[5]["inst"]], block_size=bs, elems_per_thread=ept).launch()
    for key in ("s", "mn", "mx", "y"):
        got = again[5][key].data_ro
        np.testing.assert_array_equal(got, mix[5][key].data_ro)


def test_batch_signature_mismatch_raises(op2):
    from pyop2_b200 import batch
    a = _direct_instances(op2, [10], 0)[0]["inst"]
    st = op2.Set(10, 1)
    d = op2.Dat(st, np.zeros(10), np.float64)
    other = batch.LoopInstance(op2.Kernel("void z(double *a) { a[0] = 1.0; }", "z"), st,
                               d(op2.IdentityMap, op2.WRITE))
    with pytest.raises(ValueError):
        batch.BatchLoop([a, other])
    with pytest.raises(ValueError):
        batch.BatchLoop([])


def _p1_instances(api, n_list, seed):
    """P1 mass Mat + RHS on several permuted structured meshes."""
    out = []
    for j, (nx, ny) in enumerate(n_list):
        coords, elem = meshes.rect_p1(nx, ny, seed=seed + j)
        P = fem.build_p1(api, 0, coords=coords, elem=elem, stiffness=True)
        out.append(P)
    return out


def test_p1_batch_matches_plain_and_oracle(op2):
    from pyop2_b200 import batch
    shapes = [(3, 40), (17, 9), (64, 64), (1, 1), (120, 7)]
    G = _p1_instances(op2, shapes, 3)
    mass = [batch.LoopInstance(P.k_mass, P.elements(3, 3),
                               P.mat((P.elem_node[op2.i[0]], P.elem_node[op2.i[1]]), op2.INC),
                               P.coords(P.elem_vnode, op2.READ)) for P in G]
    rhs = [batch.LoopInstance(P.k_rhs, P.elements(3), P.b(P.elem_node[op2.i[0]], op2.INC),
                              P.coords(P.elem_vnode, op2.READ), P.f(P.elem_node, op2.READ))
           for P in G]
    stiff = [batch.LoopInstance(P.k_stiff, P.elements(3, 3),
                                P.stiff((P.elem_node[op2.i[0]], P.elem_node[op2.i[1]]), op2.INC),
                                P.coords(P.elem_vnode, op2.READ)) for P in G]
    batch.BatchLoop(mass, block_size=128, elems_per_thread=2).launch()
    batch.BatchLoop(rhs, block_size=256).launch()
    batch.BatchLoop(stiff, block_size=512, elems_per_thread=4).launch()
    O = _p1_instances(seq, shapes, 3)
    for P, Q in zip(G, O):
        fem.assemble_p1(seq, Q)
        fem.assemble_p1_stiffness(seq, Q)
        np.testing.assert_array_equal(P.sparsity._rowptr, Q.sparsity.rowptr)
        assert rel_err(P.mat.array, Q.mat.array) < TOL
        assert rel_err(P.stiff.array, Q.stiff.array) < TOL
        assert rel_err(P.b.data_ro, Q.b.data) < TOL


def test_autotuned_batch_and_graph_replay(op2):
    """The tuner times its candidates and returns one of them; the tuned
    batch recorded in a CUDA graph gives the plain path's results."""
    from pyop2_b200 import autotune, b200, batch
    from pyop2_b200.workloads import batching
    shapes = batching.mesh_shapes(12, seed=5)
    G = batching.build(op2, shapes, seed=5)
    mass, stiff, rhs = batching.instances(op2, G)
    cands = (dict(block_size=128, elems_per_thread=1, min_blocks=0, ctas_per_sm=0),
             dict(block_size=256, elems_per_thread=2, min_blocks=0, ctas_per_sm=2))
    loops = []
    for insts in (mass, stiff, rhs):
        best, times = autotune.tune(insts, candidates=cands, reps=2, use_cache=False)
        assert best in [dict(c) for c in cands] and len(times) == 2
        loops.append(autotune.build(insts, best))
    for P in G:
        P.mat.zero(); P.stiff.zero(); P.b.zero()
    for bl in loops:
        bl.launch()
    b200.synchronize()
    with b200.capture() as g:
        for bl in loops:
            bl.launch(sync_host=False)
    for P in G:
        P.mat.zero(); P.stiff.zero(); P.b.zero()
    g.launch()
    got = [(P.mat.array.copy(), P.stiff.array.copy(), P.b.data_ro.copy()) for P in G]
    g.close()
    for P, (m, k, b) in zip(G, got):
        P.mat.zero(); P.stiff.zero(); P.b.zero()
        batching.plain(op2, P)
        assert rel_err(m, P.mat.array) < TOL
        assert rel_err(k, P.stiff.array) < TOL
        assert rel_err(b, P.b.data_ro) < TOL


@pytest.mark.parametrize("part_size,bs", [(128, 128), (512, 256)])
def test_coloured_batch_matches_oracle(op2, part_size, bs):
    """The coloured batched form: every mesh carries its own plan (blocks of
    ``part_size`` elements, block colours, thread colours), each launch runs
    one block colour of every mesh; Mats and the RHS against the oracle."""
    from pyop2_b200 import b200, batch
    from pyop2_b200.workloads import batching
    shapes = batching.mesh_shapes(24, seed=8)
    G = batching.build(op2, shapes, seed=8)
    loops = [batch.BatchLoop([i.recast("color", part_size) for i in insts], block_size=bs)
             for insts in batching.instances(op2, G)]
    assert all(bl.form == "color" and bl.launches >= 1 for bl in loops)
    for P in G:
        P.mat.zero(); P.stiff.zero(); P.b.zero()
    for bl in loops:
        bl.launch()
    b200.synchronize()
    for P in G:
        Q = fem.build_p1(seq, 0, coords=P.coords.data_ro, elem=P.elem_node.values, stiffness=True)
        fem.assemble_p1(seq, Q)
        fem.assemble_p1_stiffness(seq, Q)
        assert rel_err(P.mat.array, Q.mat.array) < TOL
        assert rel_err(P.stiff.array, Q.stiff.array) < TOL
        assert rel_err(P.b.data_ro, Q.b.data) < TOL
