"""The sequential oracle on the cases of the reference's unit tests whose
answers are exact: vector-map and iteration-space access to Dats (READ,
WRITE, INC of 1- and 2-component rows through a 2-to-1 node-to-element Map;
test/unit/test_vector_map.py and test_iteration_space_dats.py) and Global
MIN / MAX / INC reductions over 4096 elements of several types
(test/unit/test_global_reduction.py).  The expected values are the ones
those tests state.  CPU only."""

import numpy as np
import pytest

from conftest import py2_shuffle, reference_seed
from oracle import seq

NNODES = 4096
NELE = NNODES // 2


def _node2ele(dim):
    node, ele = seq.Set(NNODES, dim, "node"), seq.Set(NELE, dim, "ele")
    return node, ele, seq.Map(node, ele, 1, np.arange(NNODES) // 2, "node2ele")


def _arg(vd, m, acc, itspace):
    return vd(m[seq.i[0]], acc) if itspace else vd(m, acc)


def _sig(itspace, dim):
    """Kernel parameter for the element row: a pointer, or (vector Map) an
    array of one row pointer."""
    return ("int *vd", "vd[%d]") if itspace else ("int *vd[1]", "vd[0][%d]")


def _loop(code, node, itspace, *args):
    seq.par_loop(seq.Kernel(code, "k"), node(1) if itspace else node, *args)


@pytest.mark.parametrize("itspace", [False, True])
def test_sum_nodes_to_edges(itspace):
    nedges = NNODES - 1
    nodes, edges = seq.Set(NNODES, 1, "nodes"), seq.Set(nedges, 1, "edges")
    node_vals = seq.Dat(nodes, np.arange(NNODES, dtype=np.uint32), np.uint32, "node_vals")
    edge_vals = seq.Dat(edges, np.zeros(nedges, dtype=np.uint32), np.uint32, "edge_vals")
    e2n = seq.Map(edges, nodes, 2, np.array([(i, i + 1) for i in range(nedges)]), "edge2node")
    if itspace:
        code = "void k(unsigned int *nodes, unsigned int *edge, int i) { *edge += nodes[0]; }"
        seq.par_loop(seq.Kernel(code, "k"), edges(2), node_vals(e2n[seq.i[0]], seq.READ),
                     edge_vals(seq.IdentityMap, seq.INC))
    else:
        code = "void k(unsigned int *nodes[1], unsigned int *edge) { *edge = nodes[0][0] + nodes[1][0]; }"
        seq.par_loop(seq.Kernel(code, "k"), edges, node_vals(e2n, seq.READ),
                     edge_vals(seq.IdentityMap, seq.WRITE))
    np.testing.assert_array_equal(edge_vals.data.ravel(), np.arange(1, nedges * 2 + 1, 2))


@pytest.mark.parametrize("itspace", [False, True])
@pytest.mark.parametrize("dim", [1, 2])
def test_read_rows(itspace, dim):
    node, ele, m = _node2ele(dim)
    d = seq.Dat(node, np.zeros(NNODES * dim), np.int32)
    vd = seq.Dat(ele, np.arange(NELE * dim), np.int32)
    p, r = _sig(itspace, dim)
    body = " ".join("d[%d] = %s;" % (c, r % c) for c in range(dim))
    _loop("void k(int *d, %s%s) { %s }" % (p, ", int i" if itspace else "", body), node, itspace,
          d(seq.IdentityMap, seq.WRITE), _arg(vd, m, seq.READ, itspace))
    np.testing.assert_array_equal(d.data[::2], vd.data)
    np.testing.assert_array_equal(d.data[1::2], vd.data)


@pytest.mark.parametrize("itspace", [False, True])
@pytest.mark.parametrize("dim", [1, 2])
def test_write_rows(itspace, dim):
    node, ele, m = _node2ele(dim)
    vd = seq.Dat(ele, np.zeros(NELE * dim), np.int32)
    p, r = _sig(itspace, dim)
    body = " ".join("%s = %d;" % (r % c, 2 + c) for c in range(dim))
    _loop("void k(%s%s) { %s }" % (p, ", int i" if itspace else "", body), node, itspace,
          _arg(vd, m, seq.WRITE, itspace))
    for c in range(dim):
        assert (vd.data.reshape(NELE, dim)[:, c] == 2 + c).all()


@pytest.mark.parametrize("itspace", [False, True])
@pytest.mark.parametrize("dim", [1, 2])
def test_inc_rows(itspace, dim):
    node, ele, m = _node2ele(dim)
    d = seq.Dat(node, np.arange(NNODES * dim), np.int32)
    start = [3, 4][:dim]
    vd = seq.Dat(ele, np.tile(start, NELE), np.int32)
    p, r = _sig(itspace, dim)
    body = " ".join("%s += d[%d];" % (r % c, c) for c in range(dim))
    _loop("void k(int *d, %s%s) { %s }" % (p, ", int i" if itspace else "", body), node, itspace,
          d(seq.IdentityMap, seq.READ), _arg(vd, m, seq.INC, itspace))
    got = vd.data.reshape(NELE, dim)
    for c in range(dim):
        want = start[c] + np.arange(c, dim * NNODES, 2 * dim) + np.arange(c + dim, dim * NNODES, 2 * dim)
        np.testing.assert_array_equal(got[:, c], want)


@pytest.mark.parametrize("dtype,ctype,fill,g0,mode,want", [
    (np.uint32, "unsigned int", 12, 8, "MIN", 8),
    (np.int32, "int", -12, 8, "MIN", -12),
    (np.int32, "int", -12, -42, "MAX", -12),
    (np.uint32, "unsigned int", 12, 42, "MAX", 42),
    (np.float32, "float", -12.0, -42.0, "MAX", -12.0),
    (np.float64, "double", -12.0, 8.0, "MIN", -12.0),
    (np.uint32, "unsigned int", 12, 0, "INC", 12 * 4096),
    (np.int32, "int", -12, 0, "INC", -12 * 4096),
    (np.float64, "double", -12.0, 0.0, "INC", -12.0 * 4096),
])
def test_global_reductions(dtype, ctype, fill, g0, mode, want):
    s = seq.Set(4096, 1, "set")
    d = seq.Dat(s, [fill] * 4096, dtype, "d")
    g = seq.Global(1, g0, dtype, "g")
    op = {"MIN": "if (*x < *g) *g = *x;", "MAX": "if (*x > *g) *g = *x;", "INC": "*g += *x;"}[mode]
    seq.par_loop(seq.Kernel("void k(%s *x, %s *g) { %s }" % (ctype, ctype, op), "k"), s,
                 d(seq.IdentityMap, seq.READ), g(getattr(seq, mode)))
    assert g.data[0] == want


def test_global_two_components():
    s = seq.Set(4096, 2, "set2")
    d = seq.Dat(s, np.arange(2 * 4096) + 1, np.uint32, "d2")
    g = seq.Global(2, [0, 0], np.uint32, "g")
    seq.par_loop(seq.Kernel("void k(unsigned int *x, unsigned int *g) { g[0] += x[0]; g[1] += x[1]; }", "k"),
                 s, d(seq.IdentityMap, seq.READ), g(seq.INC))
    v = np.arange(2 * 4096) + 1
    assert g.data[0] == v[0::2].sum() and g.data[1] == v[1::2].sum()


# -------------------------------------------- direct loops (test_direct_loop.py)
def _direct(code, name, s, *args):
    seq.par_loop(seq.Kernel(code, name), s, *args)


def test_direct_loops():
    n = 4096
    elems, elems2 = seq.Set(n, 1, "elems"), seq.Set(n, 2, "elems2")
    x = seq.Dat(elems, np.arange(n, dtype=np.uint32), np.uint32, "x")
    _direct("void kernel_wo(unsigned int *x) { *x = 42; }", "kernel_wo", elems, x(seq.IdentityMap, seq.WRITE))
    assert (x.data == 42).all()
    x = seq.Dat(elems, np.arange(n, dtype=np.uint32), np.uint32, "x")
    _direct("void kernel_rw(unsigned int *x) { (*x) = (*x) + 1; }", "kernel_rw", elems,
            x(seq.IdentityMap, seq.RW))
    assert x.data.sum() == n * (n + 1) // 2
    x = seq.Dat(elems, np.arange(n, dtype=np.uint32), np.uint32, "x")
    g = seq.Global(1, 0, np.uint32, "g")
    _direct("void kgi(unsigned int *x, unsigned int *inc) { (*x) = (*x) + 1; (*inc) += (*x); }", "kgi",
            elems, x(seq.IdentityMap, seq.RW), g(seq.INC))
    assert g.data[0] == n * (n + 1) // 2
    g = seq.Global(1, 10, np.uint32, "g")
    _direct("void k1(unsigned int *inc) { (*inc) += 1; }", "k1", elems, g(seq.INC))
    assert g.data[0] == n + 10
    x = seq.Dat(elems, np.arange(n, dtype=np.uint32), np.uint32, "x")
    kmax = "void kmax(unsigned int *x, unsigned int *g) { if (*g < *x) { *g = *x; } }"
    for g0, want in ((0, n - 1), (2 * n, 2 * n)):
        g = seq.Global(1, g0, np.uint32, "g")
        _direct(kmax, "kmax", elems, x(seq.IdentityMap, seq.READ), g(seq.MAX))
        assert g.data[0] == want
    kmin = "void kmin(unsigned int *x, unsigned int *g) { if (*g > *x) { *g = *x; } }"
    g = seq.Global(1, 1000, np.uint32, "g")
    _direct(kmin, "kmin", elems, x(seq.IdentityMap, seq.READ), g(seq.MIN))
    assert g.data[0] == 0
    h = seq.Global(1, 1, np.uint32, "h")
    _direct("void kgr(unsigned int *x, unsigned int *h) { (*x) += (*h); }", "kgr", elems,
            x(seq.IdentityMap, seq.RW), h(seq.READ))
    assert x.data.sum() == n * (n + 1) // 2
    y = seq.Dat(elems2, np.zeros(2 * n, np.uint32), np.uint32, "y")
    _direct("void k2d(unsigned int *x) { x[0] = 42; x[1] = 43; }", "k2d", elems2, y(seq.IdentityMap, seq.WRITE))
    assert (y.data[:, 0] == 42).all() and (y.data[:, 1] == 43).all()
    soa = seq.Dat(elems2, np.zeros(2 * n, np.uint32), np.uint32, "soa", soa=True)
    _direct("void ksoa(unsigned int *x) { OP2_STRIDE(x, 0) = 42; OP2_STRIDE(x, 1) = 43; }", "ksoa", elems2,
            soa(seq.IdentityMap, seq.WRITE))
    assert (soa.data[:, 0] == 42).all() and (soa.data[:, 1] == 43).all()


# ---------------------------------------- indirect loops (test_indirect_loop.py)
def test_indirect_loops():
    n = 4096
    iterset, indset = seq.Set(n, 1, "iterset"), seq.Set(n, 1, "indset")
    u = np.arange(n, dtype=np.int32)
    py2_shuffle(u, reference_seed)
    m = seq.Map(iterset, indset, 1, u, "iterset2indset")

    def fresh():
        return seq.Dat(indset, np.arange(n, dtype=np.uint32), np.uint32, "x")
    x = fresh()
    _direct("void kernel_wo(unsigned int *x) { *x = 42; }", "kernel_wo", iterset, x(m[0], seq.WRITE))
    assert (x.data == 42).all()
    x = fresh()
    _direct("void kernel_rw(unsigned int *x) { (*x) = (*x) + 1; }", "kernel_rw", iterset, x(m[0], seq.RW))
    assert x.data.sum() == n * (n + 1) // 2
    unitset = seq.Set(1, 1, "unitset")
    ud = seq.Dat(unitset, np.array([0], np.uint32), np.uint32, "u")
    mu = seq.Map(iterset, unitset, 1, np.zeros(n, np.int32), "iterset2unitset")
    _direct("void kernel_inc(unsigned int *x) { (*x) = (*x) + 1; }", "kernel_inc", iterset, ud(mu[0], seq.INC))
    assert ud.data[0] == n
    x = fresh()
    g = seq.Global(1, 2, np.uint32, "g")
    _direct("void kgr(unsigned int *x, unsigned int *g) { (*x) /= (*g); }", "kgr", iterset,
            x(m[0], seq.RW), g(seq.READ))
    assert x.data.sum() == sum(v // 2 for v in range(n))
    x = fresh()
    g = seq.Global(1, 0, np.uint32, "g")
    _direct("void kgi(unsigned int *x, unsigned int *inc) { (*x) = (*x) + 1; (*inc) += (*x); }", "kgi",
            iterset, x(m[0], seq.RW), g(seq.INC))
    assert x.data.sum() == n * (n + 1) // 2 and g.data[0] == n * (n + 1) // 2
    indset2 = seq.Set(n, 2, "indset2")
    x2 = seq.Dat(indset2, np.zeros(2 * n, np.uint32), np.uint32, "x2")
    m2 = seq.Map(iterset, indset2, 1, u, "iterset2indset2")
    _direct("void k2(unsigned int *x) { x[0] = 42; x[1] = 43; }", "k2", iterset, x2(m2[0], seq.WRITE))
    assert (x2.data[:, 0] == 42).all() and (x2.data[:, 1] == 43).all()
    nedges = n - 1
    nodes, edges = seq.Set(n, 1, "nodes"), seq.Set(nedges, 1, "edges")
    nv = seq.Dat(nodes, np.arange(n, dtype=np.uint32), np.uint32, "node_vals")
    ev = seq.Dat(edges, np.zeros(nedges, np.uint32), np.uint32, "edge_vals")
    e2n = seq.Map(edges, nodes, 2, np.array([(i, i + 1) for i in range(nedges)]), "edge2node")
    _direct("void ksum(unsigned int *a, unsigned int *b, unsigned int *e) { *e = *a + *b; }", "ksum", edges,
            nv(e2n[0], seq.READ), nv(e2n[1], seq.READ), ev(seq.IdentityMap, seq.WRITE))
    np.testing.assert_array_equal(ev.data.ravel(), np.arange(1, nedges * 2 + 1, 2))


# ---------------------------------------------- Consts (test_constants.py)
@pytest.mark.parametrize("dim,vals,body", [(1, 100, "*x = myconstant;"),
                                           (2, (100, 200), "*x = myconstant[0] + myconstant[1];")])
def test_const_read(dim, vals, body):
    s = seq.Set(8)
    d = seq.Dat(s, np.zeros(8, np.int32), np.int32)
    c = seq.Const(dim, vals, "myconstant", np.int32)
    try:
        _direct("void k(int *x) { %s }" % body, "k", s, d(seq.IdentityMap, seq.WRITE))
    finally:
        c.remove_from_namespace()
    assert (d.data == np.sum(vals)).all()


def test_const_change_is_seen():
    s = seq.Set(8)
    d = seq.Dat(s, np.zeros(8, np.int32), np.int32)
    c = seq.Const(1, 10, "myconstant", np.int32)
    try:
        _direct("void k(int *x) { *x = myconstant; }", "k", s, d(seq.IdentityMap, seq.WRITE))
        assert (d.data == 10).all()
        c.data[...] = 11
        _direct("void k(int *x) { *x = myconstant; }", "k", s, d(seq.IdentityMap, seq.WRITE))
        assert (d.data == 11).all()
    finally:
        c.remove_from_namespace()
