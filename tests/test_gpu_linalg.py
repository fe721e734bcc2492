"""Device linear algebra: op2.solve (CG + Jacobi), the CSR SpMV and the Dat
arithmetic, against the reference's solve tests and the CPU oracle.

Tolerances: the reference's own (x equals the field the RHS was built from
to 1e-8 for the scalar and 1e-12 for the vector mass matrix); against the
oracle CG, the same iteration count within one and the solutions within
1e-9 relative (reduction orders differ); SpMV within 1e-14 relative;
elementwise Dat arithmetic bit for bit (the same IEEE operations)."""

import numpy as np
import pytest
from numpy.testing import assert_allclose

from conftest import rel_err
from oracle import linalg
from pyop2_b200.workloads import fem, meshes

pytestmark = pytest.mark.gpu


@pytest.fixture
def op2(backend):
    from pyop2_b200 import op2 as _op2
    return _op2


def _golden_problem(op2, g):
    class P:
        pass
    p = P()
    p.nodes = op2.Set(4, 1, "nodes")
    p.vnodes = op2.Set(4, 2, "vnodes")
    p.elements = op2.Set(2, 1, "elements")
    emap = np.asarray(g["elem_node_map"], dtype=np.uint32)
    p.elem_node = op2.Map(p.elements, p.nodes, 3, emap, "elem_node")
    p.elem_vnode = op2.Map(p.elements, p.vnodes, 3, emap, "elem_vnode")
    p.mat = op2.Mat(op2.Sparsity((p.elem_node, p.elem_node)), np.float64, "mat")
    p.vecmat = op2.Mat(op2.Sparsity((p.elem_vnode, p.elem_vnode)), np.float64, "vecmat")
    p.coords = op2.Dat(p.vnodes, np.asarray(g["coords"]), np.float64, "coords")
    p.f = op2.Dat(p.nodes, np.asarray(g["f"]), np.float64, "f")
    p.f_vec = op2.Dat(p.vnodes, np.asarray(g["f_vec"]), np.float64, "f_vec")
    p.b = op2.Dat(p.nodes, np.zeros(4), np.float64, "b")
    p.b_vec = op2.Dat(p.vnodes, np.zeros(8), np.float64, "b_vec")
    p.x = op2.Dat(p.nodes, np.zeros(4), np.float64, "x")
    p.x_vec = op2.Dat(p.vnodes, np.zeros(8), np.float64, "x_vec")
    p.K = {k: op2.Kernel(v["code"], v["name"]) for k, v in g["kernels"].items()}
    return p


def test_solve_golden(op2, golden_matrices):
    """test/unit/test_matrices.py:647-650 and 780-783: assemble the mass
    matrix and the RHS of f, solve, recover f."""
    p = _golden_problem(op2, golden_matrices)
    op2.par_loop(p.K["mass"], p.elements(3, 3), p.mat((p.elem_node[op2.i[0]], p.elem_node[op2.i[1]]),
                                                      op2.INC), p.coords(p.elem_vnode, op2.READ))
    op2.par_loop(p.K["rhs"], p.elements, p.b(p.elem_node, op2.INC), p.coords(p.elem_vnode, op2.READ),
                 p.f(p.elem_node, op2.READ))
    op2.solve(p.mat, p.x, p.b)
    assert_allclose(p.x.data, p.f.data, 1e-8)
    op2.par_loop(p.K["mass_vector_ffc"], p.elements(3, 3),
                 p.vecmat((p.elem_vnode[op2.i[0]], p.elem_vnode[op2.i[1]]), op2.INC),
                 p.coords(p.elem_vnode, op2.READ))
    op2.par_loop(p.K["rhs_ffc_vector"], p.elements, p.b_vec(p.elem_vnode, op2.INC),
                 p.coords(p.elem_vnode, op2.READ), p.f_vec(p.elem_vnode, op2.READ))
    op2.solve(p.vecmat, p.x_vec, p.b_vec)
    assert_allclose(p.x_vec.data, p.f_vec.data, 1e-12)


@pytest.mark.parametrize("jacobi", [True, False])
def test_solve_matches_oracle_cg(op2, jacobi):
    from pyop2_b200 import b200
    coords, elem = meshes.rect_p1(40, 23, seed=2)
    P = fem.build_p1(op2, 0, coords=coords, elem=elem)
    fem.assemble_p1(op2, P)
    rng = np.random.default_rng(3)
    rhs = rng.standard_normal(P.n_nodes)
    b = op2.Dat(P.nodes, rhs, np.float64, "b")
    x = op2.Dat(P.nodes, np.full(P.n_nodes, 7.0), np.float64, "x")   # ignored: x0 = 0
    s = b200.Solver(preconditioner="jacobi" if jacobi else "none", relative_tolerance=1e-10)
    s.solve(P.mat, x, b)
    rp, ci, vals = P.sparsity.rowptr, P.sparsity.colidx, P.mat.array
    xo, its, reason, hist = linalg.cg(rp, ci, vals, rhs, jacobi=jacobi, rtol=1e-10)
    assert s.reason == reason == 1
    assert abs(s.iterations - its) <= 1
    assert rel_err(x.data_ro, xo) < 1e-9
    assert rel_err(s.residual_history[:3], hist[:3]) < 1e-9
    # the solution solves the system
    assert rel_err(linalg.csr_matvec(rp, ci, vals, x.data_ro.ravel()), rhs) < 1e-7


def test_nonconvergence_raises_or_warns(op2):
    from pyop2_b200 import b200
    coords, elem = meshes.square_p1(16)
    P = fem.build_p1(op2, 16, coords=coords, elem=elem)
    fem.assemble_p1(op2, P)
    b = op2.Dat(P.nodes, np.random.default_rng(4).standard_normal(P.n_nodes), np.float64)
    x = op2.Dat(P.nodes, np.zeros(P.n_nodes), np.float64)
    with pytest.raises(RuntimeError):
        b200.Solver(maximum_iterations=2, relative_tolerance=1e-14).solve(P.mat, x, b)
    s = b200.Solver(maximum_iterations=2, relative_tolerance=1e-14, error_on_nonconvergence=False)
    with pytest.warns(UserWarning):
        s.solve(P.mat, x, b)
    assert (s.iterations, s.reason) == (2, 4)
    zero = op2.Dat(P.nodes, np.zeros(P.n_nodes), np.float64)
    s = b200.Solver()
    s.solve(P.mat, x, zero)
    assert s.iterations == 0 and not x.data_ro.any()


def test_spmv_matches_oracle(op2):
    from pyop2_b200 import b200
    from pyop2_b200._lib import call
    P = fem.build_p2(op2, 24, seed=1)
    fem.assemble_p2(op2, P)
    sp = P.sparsity
    n = sp._lsize
    xv = np.random.default_rng(5).standard_normal(n)
    xd = b200._upload(xv)
    yd = b200.DeviceBuffer(n * 8)
    y0 = np.random.default_rng(6).standard_normal(n)
    yd.from_host(y0)
    call("op2b_csr_spmv", sp._d_rowptr, sp._d_colidx, P.K._device_values().ptr, n, sp._d_nz,
         xd.ptr, yd.ptr, 2.0, -0.5, 0, 0)
    y = np.empty(n)
    yd.to_host(y)
    want = 2.0 * linalg.csr_matvec(sp.rowptr, sp.colidx, P.K.array, xv) - 0.5 * y0
    assert rel_err(y, want) < 1e-14


def test_dat_arithmetic_on_device(op2):
    rng = np.random.default_rng(7)
    s = op2.Set(1000, 2)
    a0, b0 = rng.standard_normal((1000, 2)), rng.standard_normal((1000, 2)) + 3.0
    a = op2.Dat(s, a0, np.float64)
    b = op2.Dat(s, b0, np.float64)
    np.testing.assert_array_equal((a + b).data_ro, a0 + b0)
    np.testing.assert_array_equal((a - b).data_ro, a0 - b0)
    np.testing.assert_array_equal((a * b).data_ro, a0 * b0)
    np.testing.assert_array_equal((a / b).data_ro, a0 / b0)
    np.testing.assert_array_equal((a * 2.5).data_ro, a0 * 2.5)
    c = op2.Dat(s, a0.copy(), np.float64)    # a Dat keeps the array it is given
    c += b
    c *= 0.5
    np.testing.assert_array_equal(c.data_ro, (a0 + b0) * 0.5)
    assert abs(a.norm - np.linalg.norm(a0)) <= 1e-14 * np.linalg.norm(a0)
    f = op2.Dat(s, a0.astype(np.float32), np.float32)
    np.testing.assert_array_equal((f * np.float32(3.0)).data_ro, a0.astype(np.float32) * np.float32(3.0))
    i = op2.Dat(s, np.arange(2000, dtype=np.int32).reshape(1000, 2), np.int32)
    np.testing.assert_array_equal((i + i).data_ro, 2 * np.arange(2000).reshape(1000, 2))
    # integer division keeps the host semantics of the reference
    np.testing.assert_array_equal((i / 2).data_ro, (np.arange(2000).reshape(1000, 2) / 2).astype(np.int32))
