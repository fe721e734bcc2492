"""par_loop semantics on the B200 backend: the cases of the reference's
test/unit/test_direct_loop.py, test_indirect_loop.py, test_global_reduction.py,
test_vector_map.py, test_iteration_space_dats.py and test_constants.py, with
the same inputs and expected (exact, integer) results."""

import numpy as np
import pytest
from numpy.testing import assert_allclose

from conftest import py2_shuffle, reference_seed

pytestmark = pytest.mark.gpu

NELEMS = 4096  # more than one block and more than one thread per element


@pytest.fixture
def op2(backend):
    from pyop2_b200 import op2 as _op2
    return _op2


@pytest.fixture(params=["atomic", "color", "staged"])
def indirect_mode(request):
    """Indirect loops under each INC strategy: atomic adds, the coloured
    plan, and the staged locality partition."""
    from pyop2_b200 import configuration as cfg
    old = (cfg.cfg['inc_mode'], cfg.cfg['staged_min_size'])
    cfg.configure(inc_mode=request.param, staged_min_size=0)
    yield request.param
    cfg.configure(inc_mode=old[0], staged_min_size=old[1])


# ----------------------------------------------------------- direct loops
class TestDirectLoop:
    """test_direct_loop.py:79-213"""

    @pytest.fixture
    def elems(self, op2):
        return op2.Set(NELEMS, 1, "elems")

    @pytest.fixture
    def elems2(self, op2):
        return op2.Set(NELEMS, 2, "elems2")

    @pytest.fixture
    def x(self, op2, elems):
        return op2.Dat(elems, np.arange(NELEMS, dtype=np.uint32), np.uint32, "x")

    @pytest.fixture
    def y(self, op2, elems2):
        return op2.Dat(elems2, [np.arange(NELEMS), np.arange(NELEMS)], np.uint32, "x")

    @pytest.fixture
    def g(self, op2):
        return op2.Global(1, 0, np.uint32, "g")

    @pytest.fixture
    def h(self, op2):
        return op2.Global(1, 1, np.uint32, "h")

    @pytest.fixture
    def soa(self, op2, elems2):
        return op2.Dat(elems2, [np.arange(NELEMS), np.arange(NELEMS)], np.uint32, "x", soa=True)

    def test_wo(self, op2, elems, x):
        k = "void kernel_wo(unsigned int* x) { *x = 42; }"
        op2.par_loop(op2.Kernel(k, "kernel_wo"), elems, x(op2.IdentityMap, op2.WRITE))
        assert all(x.data == 42)

    def test_rw(self, op2, elems, x):
        k = "void kernel_rw(unsigned int* x) { (*x) = (*x) + 1; }"
        op2.par_loop(op2.Kernel(k, "kernel_rw"), elems, x(op2.IdentityMap, op2.RW))
        assert sum(x.data) == NELEMS * (NELEMS + 1) // 2

    def test_global_inc(self, op2, elems, x, g):
        k = "void kernel_global_inc(unsigned int* x, unsigned int* inc) { (*x) = (*x) + 1; (*inc) += (*x); }"
        op2.par_loop(op2.Kernel(k, "kernel_global_inc"), elems, x(op2.IdentityMap, op2.RW), g(op2.INC))
        assert g.data[0] == NELEMS * (NELEMS + 1) // 2

    def test_global_inc_init_not_zero(self, op2, elems, g):
        k = "void k(unsigned int* inc) { (*inc) += 1; }"
        g.data[0] = 10
        op2.par_loop(op2.Kernel(k, 'k'), elems, g(op2.INC))
        assert g.data[0] == elems.size + 10

    def test_global_max_dat_is_max(self, op2, elems, x, g):
        k = "void k(unsigned int *x, unsigned int *g) { if ( *g < *x ) { *g = *x; } }"
        op2.par_loop(op2.Kernel(k, 'k'), elems, x(op2.IdentityMap, op2.READ), g(op2.MAX))
        assert g.data[0] == x.data.max()

    def test_global_max_g_is_max(self, op2, elems, x, g):
        k = "void k(unsigned int *x, unsigned int *g) { if ( *g < *x ) { *g = *x; } }"
        g.data[0] = NELEMS * 2
        op2.par_loop(op2.Kernel(k, 'k'), elems, x(op2.IdentityMap, op2.READ), g(op2.MAX))
        assert g.data[0] == NELEMS * 2

    def test_global_min_dat_is_min(self, op2, elems, x, g):
        k = "void k(unsigned int *x, unsigned int *g) { if ( *g > *x ) { *g = *x; } }"
        g.data[0] = 1000
        op2.par_loop(op2.Kernel(k, 'k'), elems, x(op2.IdentityMap, op2.READ), g(op2.MIN))
        assert g.data[0] == x.data.min()

    def test_global_min_g_is_min(self, op2, elems, x, g):
        k = "void k(unsigned int *x, unsigned int *g) { if ( *g > *x ) { *g = *x; } }"
        g.data[0] = 10
        x.data[:] = 11
        op2.par_loop(op2.Kernel(k, 'k'), elems, x(op2.IdentityMap, op2.READ), g(op2.MIN))
        assert g.data[0] == 10

    def test_global_read(self, op2, elems, x, h):
        k = "void kernel_global_read(unsigned int* x, unsigned int* h) { (*x) += (*h); }"
        op2.par_loop(op2.Kernel(k, "kernel_global_read"), elems, x(op2.IdentityMap, op2.RW), h(op2.READ))
        assert sum(x.data) == NELEMS * (NELEMS + 1) // 2

    def test_2d_dat(self, op2, elems, y):
        k = "void kernel_2d_wo(unsigned int* x) { x[0] = 42; x[1] = 43; }"
        op2.par_loop(op2.Kernel(k, "kernel_2d_wo"), elems, y(op2.IdentityMap, op2.WRITE))
        assert all((y.data == [42, 43]).all(axis=1))

    def test_2d_dat_soa(self, op2, elems, soa):
        k = "void kernel_soa(unsigned int * x) { OP2_STRIDE(x, 0) = 42; OP2_STRIDE(x, 1) = 43; }"
        op2.par_loop(op2.Kernel(k, "kernel_soa"), elems, soa(op2.IdentityMap, op2.WRITE))
        assert all(soa.data[:, 0] == 42) and all(soa.data[:, 1] == 43)

    def test_soa_should_stay_c_contigous(self, op2, elems, soa):
        k = "void dummy(unsigned int *x) {}"
        assert soa.data.flags['C_CONTIGUOUS']
        op2.par_loop(op2.Kernel(k, "dummy"), elems, soa(op2.IdentityMap, op2.WRITE))
        assert soa.data.flags['C_CONTIGUOUS']

    def test_parloop_should_set_ro_flag(self, op2, elems, x):
        k = "void k(unsigned int *x) { *x = 1; }"
        x_data = x.data
        op2.par_loop(op2.Kernel(k, 'k'), elems, x(op2.IdentityMap, op2.WRITE))
        with pytest.raises((RuntimeError, ValueError)):
            x_data[0] = 1

    def test_host_write_works(self, op2, elems, x, g):
        k = "void k(unsigned int *x, unsigned int *g) { *g += *x; }"
        x.data[:] = 1
        g.data[:] = 0
        op2.par_loop(op2.Kernel(k, 'k'), elems, x(op2.IdentityMap, op2.READ), g(op2.INC))
        assert g.data[0] == NELEMS
        x.data[:] = 2
        g.data[:] = 0
        op2.par_loop(op2.Kernel(k, 'k'), elems, x(op2.IdentityMap, op2.READ), g(op2.INC))
        assert g.data[0] == 2 * NELEMS

    def test_zero_1d_dat_works(self, op2, x):
        x.data[:] = 10
        assert (x.data == 10).all()
        x.zero()
        assert (x.data == 0).all()

    def test_zero_2d_dat_works(self, op2, y):
        y.data[:] = 10
        assert (y.data == 10).all()
        y.zero()
        assert (y.data == 0).all()

    def test_empty_set(self, op2):
        s = op2.Set(0, 1, "empty")
        d = op2.Dat(s, np.zeros(0), np.float64, "d")
        g = op2.Global(1, 3.0, np.float64, "g")
        op2.par_loop(op2.Kernel("void k(double *x, double *g) { *g += *x; }", "k"), s,
                     d(op2.IdentityMap, op2.READ), g(op2.INC))
        assert g.data[0] == 3.0

    def test_ragged_sizes(self, op2):
        for n in (1, 31, 33, 255, 257, 1000003):
            s = op2.Set(n, 3, "s")
            d = op2.Dat(s, np.arange(3 * n, dtype=np.float64), np.float64, "d")
            g = op2.Global(1, 0.0, np.float64, "g")
            op2.par_loop(op2.Kernel("void k(double *x, double *g) { x[2] = x[0] + x[1]; *g += x[2]; }", "k"),
                         s, d(op2.IdentityMap, op2.RW), g(op2.INC))
            a = np.arange(3 * n, dtype=np.float64).reshape(n, 3)
            assert (d.data[:, 2] == a[:, 0] + a[:, 1]).all()
            assert_allclose(g.data[0], (a[:, 0] + a[:, 1]).sum(), rtol=1e-13)


# --------------------------------------------------------- indirect loops
class TestIndirectLoop:
    """test_indirect_loop.py:70-145"""

    @pytest.fixture(autouse=True)
    def _mode(self, indirect_mode):
        return indirect_mode

    @pytest.fixture
    def iterset(self, op2):
        return op2.Set(NELEMS, 1, "iterset")

    @pytest.fixture
    def indset(self, op2):
        return op2.Set(NELEMS, 1, "indset")

    @pytest.fixture
    def x(self, op2, indset):
        return op2.Dat(indset, list(range(NELEMS)), np.uint32, "x")

    @pytest.fixture
    def iterset2indset(self, op2, iterset, indset):
        u_map = np.array(range(NELEMS), dtype=np.uint32)
        py2_shuffle(u_map, reference_seed)
        return op2.Map(iterset, indset, 1, u_map, "iterset2indset")

    def test_onecolor_wo(self, op2, iterset, x, iterset2indset):
        k = "void kernel_wo(unsigned int* x) { *x = 42; }\n"
        op2.par_loop(op2.Kernel(k, "kernel_wo"), iterset, x(iterset2indset[0], op2.WRITE))
        assert all(x.data == 42)

    def test_onecolor_rw(self, op2, iterset, x, iterset2indset):
        k = "void kernel_rw(unsigned int* x) { (*x) = (*x) + 1; }\n"
        op2.par_loop(op2.Kernel(k, "kernel_rw"), iterset, x(iterset2indset[0], op2.RW))
        assert sum(x.data) == NELEMS * (NELEMS + 1) // 2

    def test_indirect_inc(self, op2, iterset):
        unitset = op2.Set(1, 1, "unitset")
        u = op2.Dat(unitset, np.array([0], dtype=np.uint32), np.uint32, "u")
        iterset2unit = op2.Map(iterset, unitset, 1, np.zeros(NELEMS, dtype=np.uint32), "iterset2unitset")
        k = "void kernel_inc(unsigned int* x) { (*x) = (*x) + 1; }\n"
        op2.par_loop(op2.Kernel(k, "kernel_inc"), iterset, u(iterset2unit[0], op2.INC))
        assert u.data[0] == NELEMS

    def test_global_read(self, op2, iterset, x, iterset2indset):
        g = op2.Global(1, 2, np.uint32, "g")
        k = "void kernel_global_read(unsigned int* x, unsigned int* g) { (*x) /= (*g); }\n"
        op2.par_loop(op2.Kernel(k, "kernel_global_read"), iterset, x(iterset2indset[0], op2.RW), g(op2.READ))
        assert sum(x.data) == sum(v // 2 for v in range(NELEMS))

    def test_global_inc(self, op2, iterset, x, iterset2indset):
        g = op2.Global(1, 0, np.uint32, "g")
        k = "void kernel_global_inc(unsigned int *x, unsigned int *inc) { (*x) = (*x) + 1; (*inc) += (*x); }\n"
        op2.par_loop(op2.Kernel(k, "kernel_global_inc"), iterset, x(iterset2indset[0], op2.RW), g(op2.INC))
        assert sum(x.data) == NELEMS * (NELEMS + 1) // 2
        assert g.data[0] == NELEMS * (NELEMS + 1) // 2

    def test_2d_dat(self, op2, iterset, iterset2indset):
        indset = op2.Set(NELEMS, 2, "indset2")
        x = op2.Dat(indset, np.array([range(NELEMS), range(NELEMS)], dtype=np.uint32), np.uint32, "x")
        k = "void kernel_wo(unsigned int* x) { x[0] = 42; x[1] = 43; }\n"
        m = op2.Map(iterset, indset, 1, iterset2indset.values, "m2")
        op2.par_loop(op2.Kernel(k, "kernel_wo"), iterset, x(m[0], op2.WRITE))
        assert all((x.data == [42, 43]).all(axis=1))

    def test_2d_map(self, op2):
        nedges = NELEMS - 1
        nodes = op2.Set(NELEMS, 1, "nodes")
        edges = op2.Set(nedges, 1, "edges")
        node_vals = op2.Dat(nodes, np.arange(NELEMS, dtype=np.uint32), np.uint32, "node_vals")
        edge_vals = op2.Dat(edges, np.zeros(nedges, dtype=np.uint32), np.uint32, "edge_vals")
        e_map = np.array([(i, i + 1) for i in range(nedges)], dtype=np.uint32)
        edge2node = op2.Map(edges, nodes, 2, e_map, "edge2node")
        k = """void kernel_sum(unsigned int *nodes1, unsigned int *nodes2, unsigned int *edge)
        { *edge = *nodes1 + *nodes2; }"""
        op2.par_loop(op2.Kernel(k, "kernel_sum"), edges, node_vals(edge2node[0], op2.READ),
                     node_vals(edge2node[1], op2.READ), edge_vals(op2.IdentityMap, op2.WRITE))
        expected = np.arange(1, nedges * 2 + 1, 2).reshape(nedges, 1)
        assert (expected == edge_vals.data).all()

    def test_map_value_out_of_range_is_rejected(self, op2):
        from pyop2_b200.exceptions import MapValueError
        a, b = op2.Set(8), op2.Set(4)
        m = op2.Map(a, b, 1, np.array([0, 1, 2, 3, 4, 0, 1, 2], np.int32), "bad")
        d = op2.Dat(b, np.zeros(4), np.float64, "d")
        with pytest.raises(MapValueError):
            op2.par_loop(op2.Kernel("void k(double *x) { *x += 1.0; }", "k"), a, d(m[0], op2.INC))


# ------------------------------------------------------ Global reductions
class TestGlobalReductions:
    """test_global_reduction.py:146-400"""

    @pytest.fixture
    def set1(self, op2):
        return op2.Set(NELEMS, 1, 'set')

    @pytest.fixture
    def set2(self, op2):
        return op2.Set(NELEMS, 2, 'set2')

    @pytest.fixture
    def d1(self, op2, set1):
        return op2.Dat(set1, np.arange(NELEMS) + 1, dtype=np.uint32)

    @pytest.fixture
    def d2(self, op2, set2):
        return op2.Dat(set2, np.arange(2 * NELEMS) + 1, dtype=np.uint32)

    K1_INC = "void k(unsigned int *x, unsigned int *g) { *g += *x; }"
    K1_MIN = "void k(unsigned int *x, unsigned int *g) { if (*x < *g) *g = *x; }"
    K1_MAX = "void k(unsigned int *x, unsigned int *g) { if (*x > *g) *g = *x; }"
    K2_INC = "void k(unsigned int *x, unsigned int *g) { g[0] += x[0]; g[1] += x[1]; }"
    K2_MIN = ("void k(unsigned int *x, unsigned int *g) { if (x[0] < g[0]) g[0] = x[0];"
              " if (x[1] < g[1]) g[1] = x[1]; }")
    K2_MAX = ("void k(unsigned int *x, unsigned int *g) { if (x[0] > g[0]) g[0] = x[0];"
              " if (x[1] > g[1]) g[1] = x[1]; }")

    @pytest.mark.parametrize("dtype,ctype,init,val,acc,expect", [
        (np.uint32, "unsigned int", 8, 12, "MIN", 8),
        (np.int32, "int", 8, -12, "MIN", -12),
        (np.int32, "int", -42, -12, "MAX", -12),
        (np.float32, "float", -.8, -12.0, "MIN", -12.0),
        (np.float32, "float", -42.8, -12.0, "MAX", -12.0),
        (np.float64, "double", -.8, -12.0, "MIN", -12.0),
        (np.float64, "double", -42.8, -12.0, "MAX", -12.0)])
    def test_direct_min_max_types(self, op2, set1, dtype, ctype, init, val, acc, expect):
        d = op2.Dat(set1, [val] * NELEMS, dtype, "d")
        op = "<" if acc == "MIN" else ">"
        k = "void kr(%s* x, %s* g) { if ( *x %s *g ) *g = *x; }" % (ctype, ctype, op)
        g = op2.Global(1, init, dtype, "g")
        op2.par_loop(op2.Kernel(k, "kr"), set1, d(op2.IdentityMap, op2.READ), g(getattr(op2, acc)))
        assert_allclose(g.data[0], expect)

    def test_1d_read(self, op2, set1, d1):
        g = op2.Global(1, 1, dtype=np.uint32)
        op2.par_loop(op2.Kernel("void k(unsigned int *x, unsigned int *g) { *x = *g; }", "k"), set1,
                     d1(op2.IdentityMap, op2.WRITE), g(op2.READ))
        assert all(d1.data == g.data)

    def test_2d_read(self, op2, set1, d1):
        g = op2.Global(2, (1, 2), dtype=np.uint32)
        op2.par_loop(op2.Kernel("void k(unsigned int *x, unsigned int *g) { *x = g[0] + g[1]; }", "k"),
                     set1, d1(op2.IdentityMap, op2.WRITE), g(op2.READ))
        assert all(d1.data == g.data.sum())

    def test_1d_inc(self, op2, set1, d1):
        g = op2.Global(1, 0, dtype=np.uint32)
        op2.par_loop(op2.Kernel(self.K1_INC, "k"), set1, d1(op2.IdentityMap, op2.READ), g(op2.INC))
        assert g.data == d1.data.sum()

    def test_1d_min_dat_is_min(self, op2, set1, d1):
        g = op2.Global(1, d1.data.min() + 1, dtype=np.uint32)
        op2.par_loop(op2.Kernel(self.K1_MIN, "k"), set1, d1(op2.IdentityMap, op2.READ), g(op2.MIN))
        assert g.data == d1.data.min()

    def test_1d_min_global_is_min(self, op2, set1, d1):
        d1.data[:] += 10
        val = d1.data.min() - 1
        g = op2.Global(1, val, dtype=np.uint32)
        op2.par_loop(op2.Kernel(self.K1_MIN, "k"), set1, d1(op2.IdentityMap, op2.READ), g(op2.MIN))
        assert g.data == val

    def test_1d_max_dat_is_max(self, op2, set1, d1):
        g = op2.Global(1, d1.data.max() - 1, dtype=np.uint32)
        op2.par_loop(op2.Kernel(self.K1_MAX, "k"), set1, d1(op2.IdentityMap, op2.READ), g(op2.MAX))
        assert g.data == d1.data.max()

    def test_1d_max_global_is_max(self, op2, set1, d1):
        val = d1.data.max() + 1
        g = op2.Global(1, val, dtype=np.uint32)
        op2.par_loop(op2.Kernel(self.K1_MAX, "k"), set1, d1(op2.IdentityMap, op2.READ), g(op2.MAX))
        assert g.data == val

    def test_2d_inc(self, op2, set1, d2):
        g = op2.Global(2, (0, 0), dtype=np.uint32)
        op2.par_loop(op2.Kernel(self.K2_INC, "k"), set1, d2(op2.IdentityMap, op2.READ), g(op2.INC))
        assert g.data[0] == d2.data[:, 0].sum()
        assert g.data[1] == d2.data[:, 1].sum()

    def test_2d_min_dat_is_min(self, op2, set1, d2):
        g = op2.Global(2, (d2.data[:, 0].min() + 1, d2.data[:, 1].min() + 1), dtype=np.uint32)
        op2.par_loop(op2.Kernel(self.K2_MIN, "k"), set1, d2(op2.IdentityMap, op2.READ), g(op2.MIN))
        assert g.data[0] == d2.data[:, 0].min()
        assert g.data[1] == d2.data[:, 1].min()

    def test_2d_min_global_is_min(self, op2, set1, d2):
        d2.data[:, 0] += 10
        d2.data[:, 1] += 10
        v0, v1 = d2.data[:, 0].min() - 1, d2.data[:, 1].min() - 1
        g = op2.Global(2, (v0, v1), dtype=np.uint32)
        op2.par_loop(op2.Kernel(self.K2_MIN, "k"), set1, d2(op2.IdentityMap, op2.READ), g(op2.MIN))
        assert g.data[0] == v0 and g.data[1] == v1

    def test_2d_max_dat_is_max(self, op2, set1, d2):
        g = op2.Global(2, (d2.data[:, 0].max() - 1, d2.data[:, 1].max() - 1), dtype=np.uint32)
        op2.par_loop(op2.Kernel(self.K2_MAX, "k"), set1, d2(op2.IdentityMap, op2.READ), g(op2.MAX))
        assert g.data[0] == d2.data[:, 0].max()
        assert g.data[1] == d2.data[:, 1].max()

    def test_2d_max_global_is_max(self, op2, set1, d2):
        v0, v1 = d2.data[:, 0].max() + 1, d2.data[:, 1].max() + 1
        g = op2.Global(2, (v0, v1), dtype=np.uint32)
        op2.par_loop(op2.Kernel(self.K2_MAX, "k"), set1, d2(op2.IdentityMap, op2.READ), g(op2.MAX))
        assert g.data[0] == v0 and g.data[1] == v1

    def test_1d_multi_inc_same_global(self, op2, set1, d1):
        g = op2.Global(1, 0, dtype=np.uint32)
        k = op2.Kernel(self.K1_INC, "k")
        op2.par_loop(k, set1, d1(op2.IdentityMap, op2.READ), g(op2.INC))
        assert g.data == d1.data.sum()
        op2.par_loop(k, set1, d1(op2.IdentityMap, op2.READ), g(op2.INC))
        assert g.data == d1.data.sum() * 2

    def test_1d_multi_inc_same_global_reset(self, op2, set1, d1):
        g = op2.Global(1, 0, dtype=np.uint32)
        k = op2.Kernel(self.K1_INC, "k")
        op2.par_loop(k, set1, d1(op2.IdentityMap, op2.READ), g(op2.INC))
        assert g.data == d1.data.sum()
        g.data = 10
        op2.par_loop(k, set1, d1(op2.IdentityMap, op2.READ), g(op2.INC))
        assert g.data == d1.data.sum() + 10

    def test_1d_multi_inc_diff_global(self, op2, set1, d1):
        g = op2.Global(1, 0, dtype=np.uint32)
        g2 = op2.Global(1, 10, dtype=np.uint32)
        k = op2.Kernel(self.K1_INC, "k")
        op2.par_loop(k, set1, d1(op2.IdentityMap, op2.READ), g(op2.INC))
        assert g.data == d1.data.sum()
        op2.par_loop(k, set1, d1(op2.IdentityMap, op2.READ), g2(op2.INC))
        assert g2.data == d1.data.sum() + 10

    def test_fp64_sum_deterministic(self, op2):
        n = 3_000_001
        s = op2.Set(n)
        rng = np.random.default_rng(7)
        d = op2.Dat(s, rng.standard_normal(n), np.float64, "d")
        k = op2.Kernel("void k(double *x, double *g) { *g += *x; }", "k")
        vals = []
        for _ in range(3):
            g = op2.Global(1, 0.0, np.float64, "g")
            op2.par_loop(k, s, d(op2.IdentityMap, op2.READ), g(op2.INC))
            vals.append(g.data[0])
        assert vals[0] == vals[1] == vals[2]
        assert abs(vals[0] - np.sum(d.data_ro)) <= 1e-12 * np.abs(d.data_ro).sum()


# --------------------------------------------- vector maps / itspace Dats
NNODES = 4096
NELE = NNODES // 2


@pytest.fixture
def vm(op2):
    class VM:
        pass
    v = VM()
    v.node = op2.Set(NNODES, 1, 'node')
    v.node2 = op2.Set(NNODES, 2, 'node2')
    v.ele = op2.Set(NELE, 1, 'ele')
    v.ele2 = op2.Set(NELE, 2, 'ele2')
    v.d1 = op2.Dat(v.node, np.zeros(NNODES), dtype=np.int32)
    v.d2 = op2.Dat(v.node2, np.zeros(2 * NNODES), dtype=np.int32)
    v.vd1 = op2.Dat(v.ele, np.zeros(NELE), dtype=np.int32)
    v.vd2 = op2.Dat(v.ele2, np.zeros(2 * NELE), dtype=np.int32)
    v.node2ele = op2.Map(v.node, v.ele, 1, np.arange(NNODES) // 2, 'node2ele')
    v.node2ele2 = op2.Map(v.node2, v.ele2, 1, np.arange(NNODES) // 2, 'node2ele2')
    return v


class TestVectorMap:
    """test_vector_map.py:95-211"""

    @pytest.fixture(autouse=True)
    def _mode(self, indirect_mode):
        return indirect_mode

    def test_sum_nodes_to_edges(self, op2):
        nedges = NNODES - 1
        nodes = op2.Set(NNODES, 1, "nodes")
        edges = op2.Set(nedges, 1, "edges")
        node_vals = op2.Dat(nodes, np.arange(NNODES, dtype=np.uint32), np.uint32, "node_vals")
        edge_vals = op2.Dat(edges, np.zeros(nedges, dtype=np.uint32), np.uint32, "edge_vals")
        e_map = np.array([(i, i + 1) for i in range(nedges)], dtype=np.uint32)
        edge2node = op2.Map(edges, nodes, 2, e_map, "edge2node")
        k = "void kernel_sum(unsigned int* nodes[1], unsigned int *edge) { *edge = nodes[0][0] + nodes[1][0]; }"
        op2.par_loop(op2.Kernel(k, "kernel_sum"), edges, node_vals(edge2node, op2.READ),
                     edge_vals(op2.IdentityMap, op2.WRITE))
        assert (np.arange(1, nedges * 2 + 1, 2).reshape(nedges, 1) == edge_vals.data).all()

    def test_read_1d_vector_map(self, op2, vm):
        vm.vd1.data[:] = np.arange(NELE).reshape(NELE, 1)
        k = "void k(int *d, int *vd[1]) { *d = vd[0][0]; }"
        op2.par_loop(op2.Kernel(k, 'k'), vm.node, vm.d1(op2.IdentityMap, op2.WRITE),
                     vm.vd1(vm.node2ele, op2.READ))
        assert all(vm.d1.data[::2] == vm.vd1.data)
        assert all(vm.d1.data[1::2] == vm.vd1.data)

    def test_write_1d_vector_map(self, op2, vm):
        k = "void k(int *vd[1]) { vd[0][0] = 2; }"
        op2.par_loop(op2.Kernel(k, 'k'), vm.node, vm.vd1(vm.node2ele, op2.WRITE))
        assert all(vm.vd1.data == 2)

    def test_inc_1d_vector_map(self, op2, vm):
        vm.vd1.data[:] = 3
        vm.d1.data[:] = np.arange(NNODES).reshape(vm.d1.data.shape)
        k = "void k(int *d, int *vd[1]) { vd[0][0] += *d; }"
        op2.par_loop(op2.Kernel(k, 'k'), vm.node, vm.d1(op2.IdentityMap, op2.READ),
                     vm.vd1(vm.node2ele, op2.INC))
        expected = np.full_like(vm.vd1.data, 3)
        expected += np.arange(0, NNODES, 2).reshape(expected.shape)
        expected += np.arange(1, NNODES, 2).reshape(expected.shape)
        assert all(vm.vd1.data == expected)

    def test_read_2d_vector_map(self, op2, vm):
        vm.vd2.data[:] = np.arange(NELE * 2).reshape(NELE, 2)
        k = "void k(int *d, int *vd[2]) { d[0] = vd[0][0]; d[1] = vd[0][1]; }"
        op2.par_loop(op2.Kernel(k, 'k'), vm.node2, vm.d2(op2.IdentityMap, op2.WRITE),
                     vm.vd2(vm.node2ele2, op2.READ))
        assert all(vm.d2.data[::2, 0] == vm.vd2.data[:, 0])
        assert all(vm.d2.data[::2, 1] == vm.vd2.data[:, 1])
        assert all(vm.d2.data[1::2, 0] == vm.vd2.data[:, 0])
        assert all(vm.d2.data[1::2, 1] == vm.vd2.data[:, 1])

    def test_write_2d_vector_map(self, op2, vm):
        k = "void k(int *vd[2]) { vd[0][0] = 2; vd[0][1] = 3; }"
        op2.par_loop(op2.Kernel(k, 'k'), vm.node2, vm.vd2(vm.node2ele2, op2.WRITE))
        assert all(vm.vd2.data[:, 0] == 2)
        assert all(vm.vd2.data[:, 1] == 3)

    def test_inc_2d_vector_map(self, op2, vm):
        vm.vd2.data[:, 0] = 3
        vm.vd2.data[:, 1] = 4
        vm.d2.data[:] = np.arange(2 * NNODES).reshape(vm.d2.data.shape)
        k = "void k(int *d, int *vd[2]) { vd[0][0] += d[0]; vd[0][1] += d[1]; }"
        op2.par_loop(op2.Kernel(k, 'k'), vm.node2, vm.d2(op2.IdentityMap, op2.READ),
                     vm.vd2(vm.node2ele2, op2.INC))
        e0 = 3 + np.arange(0, 2 * NNODES, 4) + np.arange(2, 2 * NNODES, 4)
        e1 = 4 + np.arange(1, 2 * NNODES, 4) + np.arange(3, 2 * NNODES, 4)
        assert all(vm.vd2.data[:, 0] == e0)
        assert all(vm.vd2.data[:, 1] == e1)


class TestIterationSpaceDats:
    """test_iteration_space_dats.py:95-211"""

    @pytest.fixture(autouse=True)
    def _mode(self, indirect_mode):
        return indirect_mode

    def test_sum_nodes_to_edges(self, op2):
        nedges = NNODES - 1
        nodes = op2.Set(NNODES, 1, "nodes")
        edges = op2.Set(nedges, 1, "edges")
        node_vals = op2.Dat(nodes, np.arange(NNODES, dtype=np.uint32), np.uint32, "node_vals")
        edge_vals = op2.Dat(edges, np.zeros(nedges, dtype=np.uint32), np.uint32, "edge_vals")
        e_map = np.array([(i, i + 1) for i in range(nedges)], dtype=np.uint32)
        edge2node = op2.Map(edges, nodes, 2, e_map, "edge2node")
        k = "void kernel_sum(unsigned int* nodes, unsigned int *edge, int i) { *edge += nodes[0]; }"
        op2.par_loop(op2.Kernel(k, "kernel_sum"), edges(edge2node.dim),
                     node_vals(edge2node[op2.i[0]], op2.READ), edge_vals(op2.IdentityMap, op2.INC))
        assert (np.arange(1, nedges * 2 + 1, 2).reshape(nedges, 1) == edge_vals.data).all()

    def test_read_1d_itspace_map(self, op2, vm):
        vm.vd1.data[:] = np.arange(NELE).reshape(NELE, 1)
        k = "void k(int *d, int *vd, int i) { d[0] = vd[0]; }"
        op2.par_loop(op2.Kernel(k, 'k'), vm.node(vm.node2ele.dim), vm.d1(op2.IdentityMap, op2.WRITE),
                     vm.vd1(vm.node2ele[op2.i[0]], op2.READ))
        assert all(vm.d1.data[::2] == vm.vd1.data)
        assert all(vm.d1.data[1::2] == vm.vd1.data)

    def test_write_1d_itspace_map(self, op2, vm):
        k = "void k(int *vd, int i) { vd[0] = 2; }"
        op2.par_loop(op2.Kernel(k, 'k'), vm.node(vm.node2ele.dim), vm.vd1(vm.node2ele[op2.i[0]], op2.WRITE))
        assert all(vm.vd1.data == 2)

    def test_inc_1d_itspace_map(self, op2, vm):
        vm.vd1.data[:] = 3
        vm.d1.data[:] = np.arange(NNODES).reshape(vm.d1.data.shape)
        k = "void k(int *d, int *vd, int i) { vd[0] += *d; }"
        op2.par_loop(op2.Kernel(k, 'k'), vm.node(vm.node2ele.dim), vm.d1(op2.IdentityMap, op2.READ),
                     vm.vd1(vm.node2ele[op2.i[0]], op2.INC))
        expected = 3 + np.arange(0, NNODES, 2) + np.arange(1, NNODES, 2)
        assert all(vm.vd1.data.ravel() == expected)

    def test_read_2d_itspace_map(self, op2, vm):
        vm.vd2.data[:] = np.arange(NELE * 2).reshape(NELE, 2)
        k = "void k(int *d, int *vd, int i) { d[0] = vd[0]; d[1] = vd[1]; }"
        op2.par_loop(op2.Kernel(k, 'k'), vm.node2(vm.node2ele2.dim), vm.d2(op2.IdentityMap, op2.WRITE),
                     vm.vd2(vm.node2ele2[op2.i[0]], op2.READ))
        assert all(vm.d2.data[::2, 0] == vm.vd2.data[:, 0])
        assert all(vm.d2.data[1::2, 1] == vm.vd2.data[:, 1])

    def test_write_2d_itspace_map(self, op2, vm):
        k = "void k(int *vd, int i) { vd[0] = 2; vd[1] = 3; }"
        op2.par_loop(op2.Kernel(k, 'k'), vm.node2(vm.node2ele2.dim), vm.vd2(vm.node2ele2[op2.i[0]], op2.WRITE))
        assert all(vm.vd2.data[:, 0] == 2)
        assert all(vm.vd2.data[:, 1] == 3)

    def test_inc_2d_itspace_map(self, op2, vm):
        vm.vd2.data[:, 0] = 3
        vm.vd2.data[:, 1] = 4
        vm.d2.data[:] = np.arange(2 * NNODES).reshape(vm.d2.data.shape)
        k = "void k(int *d, int *vd, int i) { vd[0] += d[0]; vd[1] += d[1]; }"
        op2.par_loop(op2.Kernel(k, 'k'), vm.node2(vm.node2ele2.dim), vm.d2(op2.IdentityMap, op2.READ),
                     vm.vd2(vm.node2ele2[op2.i[0]], op2.INC))
        assert all(vm.vd2.data[:, 0] == 3 + np.arange(0, 2 * NNODES, 4) + np.arange(2, 2 * NNODES, 4))
        assert all(vm.vd2.data[:, 1] == 4 + np.arange(1, 2 * NNODES, 4) + np.arange(3, 2 * NNODES, 4))


# -------------------------------------------------------------- constants
class TestConstant:
    """test_constants.py:54-117"""

    @pytest.fixture
    def cset(self, op2):
        return op2.Set(8)

    @pytest.fixture
    def dat(self, op2, cset):
        return op2.Dat(cset, np.zeros(8, dtype=np.int32))

    def test_1d_read(self, op2, cset, dat):
        c = op2.Const(1, 100, dtype=np.int32, name="myconstant")
        op2.par_loop(op2.Kernel("void kernel_1d_read(int *x) { *x = myconstant; }", "kernel_1d_read"),
                     cset, dat(op2.IdentityMap, op2.WRITE))
        c.remove_from_namespace()
        assert all(dat.data == c.data)

    def test_2d_read(self, op2, cset, dat):
        c = op2.Const(2, (100, 200), dtype=np.int32, name="myconstant")
        op2.par_loop(op2.Kernel("void kernel_2d_read(int *x) { *x = myconstant[0] + myconstant[1]; }",
                                "kernel_2d_read"), cset, dat(op2.IdentityMap, op2.WRITE))
        c.remove_from_namespace()
        assert all(dat.data == c.data.sum())

    def test_change_constant_value(self, op2, cset, dat):
        c = op2.Const(1, 10, dtype=np.int32, name="myconstant")
        k = op2.Kernel("void k(int *x) { *x = myconstant; }", 'k')
        op2.par_loop(k, cset, dat(op2.IdentityMap, op2.WRITE))
        assert all(dat.data == 10)
        c.data = 11
        op2.par_loop(k, cset, dat(op2.IdentityMap, op2.WRITE))
        c.remove_from_namespace()
        assert all(dat.data == 11)


class TestCapture:
    """Loops recorded into a CUDA graph (b200.capture) replay the recorded
    work; a Global first used inside the recording is refused."""

    def test_replay_and_fresh_global_refused(self, op2):
        from pyop2_b200 import b200
        from pyop2_b200.exceptions import DeviceError
        s = op2.Set(1000)
        x = op2.Dat(s, np.arange(1000, dtype=np.float64), np.float64)
        g = op2.Global(1, 0.0, np.float64)
        k = op2.Kernel("void kc(double *x, double *g) { x[0] += 1.0; g[0] += x[0]; }", "kc")
        op2.par_loop(k, s, x(op2.IdentityMap, op2.RW), g(op2.INC))
        with b200.capture() as graph:
            op2.par_loop(k, s, x(op2.IdentityMap, op2.RW), g(op2.INC))
        graph.launch()
        graph.launch()
        np.testing.assert_array_equal(x.data_ro.reshape(-1), np.arange(1000) + 3.0)
        fresh = op2.Global(1, 0.0, np.float64)
        with pytest.raises(DeviceError):
            with b200.capture():
                op2.par_loop(k, s, x(op2.IdentityMap, op2.RW), fresh(op2.INC))
        graph.close()


def test_read_replica_follows_writes(backend):
    """A loop that only reads a Dat through a Map reads a copy of it in
    first-use order (READ replica); writes to the Dat from the host, from
    another par_loop and by zero() are seen by the next run."""
    from pyop2_b200 import b200, op2
    from pyop2_b200 import configuration as cfg
    cfg.configure(replica_min_size=0)
    rng = np.random.default_rng(4)
    nodes, cells = op2.Set(500, 2), op2.Set(300)
    m = rng.integers(0, 500, size=(300, 3)).astype(np.int32)
    cn = op2.Map(cells, nodes, 3, m, "cn")
    x = op2.Dat(nodes, rng.standard_normal((500, 2)), np.float64, "x")
    out = op2.Dat(cells, np.zeros(300), np.float64, "out")
    k = op2.Kernel("void k(double *a, double *b, double *c, double *o) {"
                   " o[0] = a[0] * 2.0 + b[1] - c[0] * c[1]; }", "k")

    def run():
        op2.par_loop(k, cells, x(cn[0], op2.READ), x(cn[1], op2.READ), x(cn[2], op2.READ),
                     out(op2.IdentityMap, op2.WRITE))
        xv = x.data_ro
        want = xv[m[:, 0], 0] * 2.0 + xv[m[:, 1], 1] - xv[m[:, 2], 0] * xv[m[:, 2], 1]
        np.testing.assert_array_equal(out.data_ro.ravel(), want)
    run()
    bound = [bl for bl in b200.ParLoop._bound_cache.values() if bl.spec.kernel_name == "k"]
    assert bound and bound[-1].replicas
    x.data[:] = rng.standard_normal((500, 2))            # host write
    run()
    op2.par_loop(op2.Kernel("void w(double *a) { a[0] += 1.0; a[1] *= -3.0; }", "w"), nodes,
                 x(op2.IdentityMap, op2.RW))             # device write
    run()
    x.zero()
    run()


@pytest.mark.parametrize("dtype", [np.float64, np.float32, np.int32, np.uint64])
def test_reduction_initial_value_in_launch_parameters(backend, dtype):
    """A reduction Global the host has just created or set travels into the
    loop in its launch parameters (no upload); its device value is used once
    the device holds the newest copy, and always inside a recorded graph."""
    from pyop2_b200 import b200, op2
    n = 1000
    s = op2.Set(n)
    x = op2.Dat(s, np.arange(n) % 7, dtype, "x")
    ct = {np.float64: "double", np.float32: "float", np.int32: "int",
          np.uint64: "unsigned long long"}[dtype]
    k = op2.Kernel("void k(%s *a, %s *g, %s *lo, %s *hi) { g[0] += a[0]; g[1] += 1;"
                   " if (a[0] < lo[0]) lo[0] = a[0]; if (a[0] > hi[0]) hi[0] = a[0]; }"
                   % (ct, ct, ct, ct), "k")
    g = op2.Global(2, [3, 4], dtype, "g")
    lo = op2.Global(1, 5, dtype, "lo")
    hi = op2.Global(1, 2, dtype, "hi")

    def run():
        op2.par_loop(k, s, x(op2.IdentityMap, op2.READ), g(op2.INC), lo(op2.MIN), hi(op2.MAX))

    tot = int((np.arange(n) % 7).sum())
    run()                                        # fresh Globals: values from the parameters
    np.testing.assert_array_equal(g.data_ro, np.array([3 + tot, 4 + n], dtype))
    assert lo.data_ro[0] == 0 and hi.data_ro[0] == 6
    run()                                        # device copies are the newest
    np.testing.assert_array_equal(g.data_ro, np.array([3 + 2 * tot, 4 + 2 * n], dtype))
    g.data = np.array([1, 1], dtype)             # host write
    lo.data = np.array([9], dtype)
    hi.data = np.array([-1 if dtype in (np.float64, np.float32, np.int32) else 0], dtype)
    run()
    np.testing.assert_array_equal(g.data_ro, np.array([1 + tot, 1 + n], dtype))
    assert lo.data_ro[0] == 0 and hi.data_ro[0] == 6
    g.data = np.array([0, 0], dtype)
    run()
    with b200.capture() as graph:                # graph: the device value each replay
        run()
    graph.launch()
    graph.launch()
    np.testing.assert_array_equal(g.data_ro, np.array([3 * tot, 3 * n], dtype))
    graph.close()
    g.data = np.array([2, 2], dtype)
    run()
    np.testing.assert_array_equal(g.data_ro, np.array([2 + tot, 2 + n], dtype))
