"""Caches of the B200 backend, after test/unit/test_caching.py: the JIT
module of a loop signature, the GPU plan of an (iteration set, Maps) pair,
the Sparsity of a Map pair and the Kernel of a code string are built once and
reused; a different signature, Map or kernel builds a new one."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def op2(backend):
    from pyop2_b200 import op2 as _op2
    return _op2


@pytest.fixture
def mesh(op2):
    rng = np.random.default_rng(1)
    it = op2.Set(1000, 1, "it")
    nodes = op2.Set(300, 1, "nodes")
    m = op2.Map(it, nodes, 2, rng.integers(0, 300, size=2000).astype(np.int32), "m")
    m2 = op2.Map(it, nodes, 2, rng.integers(0, 300, size=2000).astype(np.int32), "m2")
    return it, nodes, m, m2


def test_same_signature_reuses_module(op2, mesh):
    from pyop2_b200 import b200
    it, nodes, m, _ = mesh
    k = op2.Kernel("void kc1(double *a, double *b) { *a += *b; }", "kc1")
    d1, d2 = op2.Dat(nodes, np.zeros(300)), op2.Dat(nodes, np.ones(300))
    e1, e2 = op2.Dat(it, np.ones(1000)), op2.Dat(it, np.ones(1000))
    op2.par_loop(k, it, d1(m[0], op2.INC), e1(op2.IdentityMap, op2.READ))
    n = len(b200._MODULES)
    op2.par_loop(k, it, d2(m[1], op2.INC), e2(op2.IdentityMap, op2.READ))   # other Dats, other index
    op2.par_loop(k, it, d1(m[0], op2.INC), e2(op2.IdentityMap, op2.READ))
    assert len(b200._MODULES) == n + 1     # only the map index changed the code
    k2 = op2.Kernel("void kc2(double *a, double *b) { *a += 2.0 * *b; }", "kc2")
    op2.par_loop(k2, it, d1(m[0], op2.INC), e1(op2.IdentityMap, op2.READ))
    assert len(b200._MODULES) == n + 2
    assert d1.data_ro.sum() == pytest.approx(1000.0 + 1000.0 + 2000.0)


def test_plan_reused_for_same_iterset_and_maps(op2, mesh):
    from pyop2_b200 import b200
    from pyop2_b200 import configuration as cfg
    it, nodes, m, m2 = mesh
    old = cfg.cfg['inc_mode']
    cfg.configure(inc_mode='color')
    try:
        k = op2.Kernel("void kp(double *a) { *a += 1.0; }", "kp")
        d1, d2 = op2.Dat(nodes, np.zeros(300)), op2.Dat(nodes, np.zeros(300))
        op2.par_loop(k, it, d1(m[0], op2.INC))
        n = len(b200._PLAN_CACHE)
        op2.par_loop(k, it, d2(m[0], op2.INC))          # other Dat, same Map: same plan
        assert len(b200._PLAN_CACHE) == n
        op2.par_loop(k, it, d1(m2[0], op2.INC))         # other Map: a new plan
        assert len(b200._PLAN_CACHE) == n + 1
        counts = np.bincount(m.values[:, 0], minlength=300)
        np.testing.assert_array_equal(d2.data_ro.reshape(-1), counts)
    finally:
        cfg.configure(inc_mode=old)


def test_sparsity_and_kernel_cached(op2, mesh):
    it, nodes, m, m2 = mesh
    s1 = op2.Sparsity((m, m))
    assert op2.Sparsity((m, m)) is s1
    assert op2.Sparsity((m, m2)) is not s1
    assert op2.Kernel("void kk(double *x) {}", "kk") is op2.Kernel("void kk(double *x) {}", "kk")


def test_new_global_each_call_reuses_bound_loop(op2, mesh):
    """A fresh Global per call (the airfoil demo's rms) hits the loop cache:
    no recompilation, and each Global receives its own reduction."""
    from pyop2_b200 import b200
    it, _, _, _ = mesh
    x = op2.Dat(it, np.arange(1000, dtype=np.float64))
    k = op2.Kernel("void kg(double *x, double *g) { *g += *x; }", "kg")
    g0 = op2.Global(1, 0.0, np.float64)
    op2.par_loop(k, it, x(op2.IdentityMap, op2.READ), g0(op2.INC))
    nb, nm = len(b200.ParLoop._bound_cache), len(b200._MODULES)
    for i in range(3):
        g = op2.Global(1, float(i), np.float64)
        op2.par_loop(k, it, x(op2.IdentityMap, op2.READ), g(op2.INC))
        assert g.data_ro[0] == 999 * 1000 / 2 + i
    assert (len(b200.ParLoop._bound_cache), len(b200._MODULES)) == (nb, nm)
