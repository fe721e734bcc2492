"""Sparsity and Mat assembly on the B200 backend against the reference's
test/unit/test_matrices.py golden values (kernels, mesh and expected matrices
from tests/golden/matrices.json) and against the CPU oracle."""

import numpy as np
import pytest
from numpy.testing import assert_allclose

pytestmark = pytest.mark.gpu


@pytest.fixture
def op2(backend):
    from pyop2_b200 import op2 as _op2
    return _op2


class Problem:
    pass


@pytest.fixture
def P(op2, golden_matrices):
    g = golden_matrices
    p = Problem()
    p.g = g
    p.nodes = op2.Set(4, 1, "nodes")
    p.vnodes = op2.Set(4, 2, "vnodes")
    p.elements = op2.Set(2, 1, "elements")
    emap = np.asarray(g["elem_node_map"], dtype=np.uint32)
    p.elem_node = op2.Map(p.elements, p.nodes, 3, emap, "elem_node")
    p.elem_vnode = op2.Map(p.elements, p.vnodes, 3, emap, "elem_vnode")
    p.mat = op2.Mat(op2.Sparsity((p.elem_node, p.elem_node), "sparsity"), np.float64, "mat")
    p.vecmat = op2.Mat(op2.Sparsity((p.elem_vnode, p.elem_vnode), "sparsity"), np.float64, "vecmat")
    p.coords = op2.Dat(p.vnodes, np.asarray(g["coords"]), np.float64, "coords")
    p.f = op2.Dat(p.nodes, np.asarray(g["f"]), np.float64, "f")
    p.f_vec = op2.Dat(p.vnodes, np.asarray(g["f_vec"]), np.float64, "f")
    p.b = op2.Dat(p.nodes, np.zeros(4), np.float64, "b")
    p.b_vec = op2.Dat(p.vnodes, np.zeros(8), np.float64, "b")
    p.g1 = op2.Global(1, 1.0, np.float64, "g")
    p.K = {k: op2.Kernel(v["code"], v["name"]) for k, v in g["kernels"].items()}
    return p


def test_build_sparsity(op2, golden_matrices):
    s = golden_matrices["sparsity"]
    elements, nodes = op2.Set(s["nelem"]), op2.Set(s["nnodes"])
    m = op2.Map(elements, nodes, 3, s["map"])
    sp = op2.Sparsity((m, m))
    assert list(sp._rowptr) == s["rowptr"]
    assert list(sp._colidx) == s["colidx"]
    assert sp.nz == s["rowptr"][-1]


def test_sparsity_null_maps(op2):
    from pyop2_b200.exceptions import MapValueError
    s = op2.Set(5)
    with pytest.raises(MapValueError):
        m = op2.Map(s, s, 1)
        op2.Sparsity((m, m))


def test_minimal_zero_mat(op2):
    code = "void zero_mat(double local_mat[1][1], int i, int j) { local_mat[i][j] = 0.0; }"
    n = 128
    s = op2.Set(n)
    m = op2.Map(s, s, 1, np.arange(n, dtype=np.uint32))
    mat = op2.Mat(op2.Sparsity((m, m)), np.float64)
    op2.par_loop(op2.Kernel(code, "zero_mat"), s(1, 1), mat((m[op2.i[0]], m[op2.i[1]]), op2.WRITE))
    assert_allclose(mat.values, np.zeros((n, n)), 1e-12)


@pytest.mark.parametrize("kernel", ["mass", "mass_ffc"])
def test_assemble_mat(op2, P, kernel):
    op2.par_loop(P.K[kernel], P.elements(3, 3), P.mat((P.elem_node[op2.i[0]], P.elem_node[op2.i[1]]), op2.INC),
                 P.coords(P.elem_vnode, op2.READ))
    assert_allclose(P.mat.values, np.asarray(P.g["expected_matrix"]), 1e-5)


def test_assemble_rhs(op2, P):
    op2.par_loop(P.K["rhs"], P.elements, P.b(P.elem_node, op2.INC), P.coords(P.elem_vnode, op2.READ),
                 P.f(P.elem_node, op2.READ))
    assert_allclose(P.b.data, np.asarray(P.g["expected_rhs"]), 1e-12)


def test_zero_matrix(op2, P):
    op2.par_loop(P.K["mass"], P.elements(3, 3), P.mat((P.elem_node[op2.i[0]], P.elem_node[op2.i[1]]), op2.INC),
                 P.coords(P.elem_vnode, op2.READ))
    P.mat.zero()
    assert_allclose(P.mat.values, np.zeros((4, 4)), 1e-14)


def test_set_matrix(op2, P):
    op2.par_loop(P.K["kernel_inc"], P.elements(3, 3),
                 P.mat((P.elem_node[op2.i[0]], P.elem_node[op2.i[1]]), op2.INC), P.g1(op2.READ))
    assert P.mat.array.sum() == 3 * 3 * P.elements.size
    op2.par_loop(P.K["kernel_set"], P.elements(3, 3),
                 P.mat((P.elem_node[op2.i[0]], P.elem_node[op2.i[1]]), op2.WRITE), P.g1(op2.READ))
    assert_allclose(P.mat.array, np.ones_like(P.mat.array))


def test_set_matrix_vec(op2, P):
    op2.par_loop(P.K["kernel_inc_vec"], P.elements(3, 3),
                 P.vecmat((P.elem_vnode[op2.i[0]], P.elem_vnode[op2.i[1]]), op2.INC), P.g1(op2.READ))
    assert P.vecmat.array.sum() == 2 * 2 * 3 * 3 * P.elements.size
    op2.par_loop(P.K["kernel_set_vec"], P.elements(3, 3),
                 P.vecmat((P.elem_vnode[op2.i[0]], P.elem_vnode[op2.i[1]]), op2.WRITE), P.g1(op2.READ))
    assert_allclose(P.vecmat.array, np.ones_like(P.vecmat.array))


def test_zero_rhs(op2, P):
    op2.par_loop(P.K["zero_dat"], P.nodes, P.b(op2.IdentityMap, op2.WRITE))
    assert (P.b.data == 0).all()


def test_assemble_vec_mass(op2, P):
    op2.par_loop(P.K["mass_vector_ffc"], P.elements(3, 3),
                 P.vecmat((P.elem_vnode[op2.i[0]], P.elem_vnode[op2.i[1]]), op2.INC),
                 P.coords(P.elem_vnode, op2.READ))
    assert_allclose(P.vecmat.values, np.asarray(P.g["expected_vector_matrix"]), 1e-6)


def test_rhs_ffc(op2, P):
    op2.par_loop(P.K["rhs_ffc"], P.elements, P.b(P.elem_node, op2.INC), P.coords(P.elem_vnode, op2.READ),
                 P.f(P.elem_node, op2.READ))
    assert_allclose(P.b.data, np.asarray(P.g["expected_rhs"]), 1e-6)


def test_rhs_ffc_itspace(op2, P):
    op2.par_loop(P.K["zero_dat"], P.nodes, P.b(op2.IdentityMap, op2.WRITE))
    op2.par_loop(P.K["rhs_ffc_itspace"], P.elements(3), P.b(P.elem_node[op2.i[0]], op2.INC),
                 P.coords(P.elem_vnode, op2.READ), P.f(P.elem_node, op2.READ))
    assert_allclose(P.b.data, np.asarray(P.g["expected_rhs"]), 1e-6)


def test_rhs_vector_ffc(op2, P):
    op2.par_loop(P.K["rhs_ffc_vector"], P.elements, P.b_vec(P.elem_vnode, op2.INC),
                 P.coords(P.elem_vnode, op2.READ), P.f_vec(P.elem_vnode, op2.READ))
    assert_allclose(P.b_vec.data, np.asarray(P.g["expected_vec_rhs"]), 1e-6)


def test_rhs_vector_ffc_itspace(op2, P):
    op2.par_loop(P.K["zero_vec_dat"], P.nodes, P.b_vec(op2.IdentityMap, op2.WRITE))
    op2.par_loop(P.K["rhs_ffc_vector_itspace"], P.elements(3), P.b_vec(P.elem_vnode[op2.i[0]], op2.INC),
                 P.coords(P.elem_vnode, op2.READ), P.f_vec(P.elem_vnode, op2.READ))
    assert_allclose(P.b_vec.data, np.asarray(P.g["expected_vec_rhs"]), 1e-6)


def test_zero_rows(op2, P):
    op2.par_loop(P.K["mass"], P.elements(3, 3), P.mat((P.elem_node[op2.i[0]], P.elem_node[op2.i[1]]), op2.INC),
                 P.coords(P.elem_vnode, op2.READ))
    expected = np.asarray(P.g["expected_matrix"])
    expected[0] = [12.0, 0.0, 0.0, 0.0]
    P.mat.zero_rows([0], 12.0)
    assert_allclose(P.mat.values, expected, 1e-5)
    expected[3] = [0.0, 0.0, 0.0, 4.0]
    P.mat.zero_rows([3], 4.0)
    assert_allclose(P.mat.values, expected, 1e-5)


def test_zero_rows_out_of_range_raises_before_launch(op2, P):
    """A row outside the matrix raises IndexError on the host (PETSc's
    zeroRowsLocal raises for the reference, pyop2/petsc_base.py:131-135) and
    leaves every value as it was."""
    op2.par_loop(P.K["mass"], P.elements(3, 3), P.mat((P.elem_node[op2.i[0]], P.elem_node[op2.i[1]]), op2.INC),
                 P.coords(P.elem_vnode, op2.READ))
    before = P.mat.array.copy()
    for rows in ([4], [0, -1], [1, 2, 99]):
        with pytest.raises(IndexError):
            P.mat.zero_rows(rows, 1.0)
    np.testing.assert_array_equal(P.mat.array, before)


def test_zero_vector_matrix(op2, P):
    P.vecmat.zero()
    assert_allclose(P.vecmat.values, np.zeros((8, 8)), 1e-14)


def test_insert_outside_sparsity_raises(op2):
    """An addto outside the pattern is an error (PETSc
    NEW_NONZERO_ALLOCATION_ERR, pyop2/petsc_base.py:113-115)."""
    from pyop2_b200.exceptions import MapValueError
    el, nd = op2.Set(2), op2.Set(4)
    m1 = op2.Map(el, nd, 2, np.array([0, 1, 2, 3], np.int32), "m1")
    m2 = op2.Map(el, nd, 2, np.array([0, 1, 2, 3], np.int32), "m2")
    mat = op2.Mat(op2.Sparsity((m1, m1)), np.float64)
    # m2 has the same values, so every entry exists: no error
    op2.par_loop(op2.Kernel("void k(double a[1][1], int i, int j) { a[0][0] = 1.0; }", "k"), el(2, 2),
                 mat((m1[op2.i[0]], m1[op2.i[1]]), op2.INC))
    assert mat.array.sum() == 8.0
    mat3 = op2.Mat(op2.Sparsity((m1, m1)), np.float64)
    m3 = op2.Map(el, nd, 2, np.array([0, 3, 2, 1], np.int32), "m3")
    sp = op2.Sparsity(((m1, m1), (m1, m3)))
    mat4 = op2.Mat(sp, np.float64)
    op2.par_loop(op2.Kernel("void k2(double a[1][1], int i, int j) { a[0][0] = 1.0; }", "k2"), el(2, 2),
                 mat4((m1[op2.i[0]], m3[op2.i[1]]), op2.INC))
    assert mat4.array.sum() == 8.0
    del mat3, m2
    with pytest.raises(MapValueError):
        from pyop2_b200 import b200
        # a Mat whose pattern lacks (0, 3): assemble through m3 columns
        sp_small = op2.Sparsity((m1, m1))
        matx = op2.Mat(sp_small, np.float64)
        loop = b200.ParLoop(op2.Kernel("void k3(double a[1][1], int i, int j) { a[0][0] = 1.0; }", "k3"),
                            el(2, 2), matx((m1[op2.i[0]], m1[op2.i[1]]), op2.INC))
        # rebind the column map behind the Arg to m3 (not in the pattern)
        loop.args[0]._map = [m1, m3]
        loop.compute()
        matx.array


def test_slot_table_matches_row_search(op2):
    """The scatter-slot table holds, for every element's (r, c) entry, the
    CSR position a row search finds; assembly through it equals assembly by
    search within the INC tolerance."""
    from pyop2_b200 import configuration as cfg
    from pyop2_b200.workloads import fem, meshes
    coords, elem = meshes.rect_p1(9, 5, seed=4)
    P = fem.build_p1(op2, 0, coords=coords, elem=elem, stiffness=True)
    sp = P.sparsity
    buf = sp._slot_table(P.elem_node, P.elem_node)
    n = len(elem)
    got = np.empty(n * 9, dtype=np.int32)
    buf.to_host(got)
    rp, ci = sp.rowptr, sp.colidx
    for e in range(n):
        for r in range(3):
            for c in range(3):
                row, col = elem[e, r], elem[e, c]
                seg = ci[rp[row]:rp[row + 1]]
                want = rp[row] + int(np.searchsorted(seg, col))
                assert got[(r * 3 + c) * n + e] == want
    vals = {}
    for slots in (True, False):
        cfg.configure(mat_slots=slots)
        try:
            P.stiff.zero()
            fem.assemble_p1_stiffness(op2, P)
            vals[slots] = P.stiff.array.copy()
        finally:
            cfg.configure(mat_slots=True)
    assert np.abs(vals[True] - vals[False]).max() <= 1e-12 * np.abs(vals[False]).max()
