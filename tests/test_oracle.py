"""The oracle, pinned: against the reference's golden vectors (Sparsity CSR,
expected mass matrices and RHS of test_matrices.py, the mass2d_triangle
regression summary) and against the reference's own compiled
build_sparsity_pattern_seq.  CPU only."""

import os

import numpy as np
import pytest
from numpy.testing import assert_allclose

from oracle import plan as oplan
from oracle import reference, seq
from pyop2_b200.workloads import meshes

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(autouse=True)
def _clean_consts():
    seq._CONSTS.clear()
    yield
    seq._CONSTS.clear()


def test_sparsity_golden(golden_matrices):
    s = golden_matrices["sparsity"]
    m = seq.Map(seq.Set(s["nelem"]), seq.Set(s["nnodes"]), 3, s["map"])
    sp = seq.Sparsity((m, m))
    assert list(sp.rowptr) == s["rowptr"]
    assert list(sp.colidx) == s["colidx"]


@pytest.mark.skipif(not reference.available(), reason="reference sparsity_utils.cxx not compiled here")
@pytest.mark.parametrize("rmult,cmult,seed", [(1, 1, 0), (2, 2, 1), (1, 3, 2)])
def test_sparsity_restatement_equals_reference(rmult, cmult, seed):
    rng = np.random.default_rng(seed)
    it, rows, cols = seq.Set(700), seq.Set(300, rmult), seq.Set(350, cmult)
    rm = seq.Map(it, rows, 3, rng.integers(0, 300, size=(700, 3)))
    cm = seq.Map(it, cols, 2, rng.integers(0, 350, size=(700, 2)))
    it2 = seq.Set(200)
    rm2 = seq.Map(it2, rows, 1, rng.integers(0, 300, size=(200, 1)))
    cm2 = seq.Map(it2, cols, 4, rng.integers(0, 350, size=(200, 4)))
    a = seq.Sparsity(((rm, cm), (rm2, cm2)))
    b = seq.Sparsity(((rm, cm), (rm2, cm2)), use_reference=True)
    np.testing.assert_array_equal(a.rowptr, b.rowptr)
    np.testing.assert_array_equal(a.colidx, b.colidx)
    np.testing.assert_array_equal(a.nnz, b.nnz)


class _Mesh:
    def __init__(self, g):
        self.nodes, self.vnodes, self.elements = seq.Set(4, 1), seq.Set(4, 2), seq.Set(2, 1)
        em = np.asarray(g["elem_node_map"])
        self.en = seq.Map(self.elements, self.nodes, 3, em)
        self.evn = seq.Map(self.elements, self.vnodes, 3, em)
        self.coords = seq.Dat(self.vnodes, np.asarray(g["coords"]))
        self.f = seq.Dat(self.nodes, np.asarray(g["f"]))
        self.f_vec = seq.Dat(self.vnodes, np.asarray(g["f_vec"]))
        self.K = {k: seq.Kernel(v["code"], v["name"]) for k, v in g["kernels"].items()}


@pytest.mark.parametrize("kernel", ["mass", "mass_ffc"])
def test_oracle_mass_golden(golden_matrices, kernel):
    M = _Mesh(golden_matrices)
    mat = seq.Mat(seq.Sparsity((M.en, M.en)))
    seq.par_loop(M.K[kernel], M.elements(3, 3), mat((M.en[seq.i[0]], M.en[seq.i[1]]), seq.INC),
                 M.coords(M.evn, seq.READ))
    assert_allclose(mat.values, np.asarray(golden_matrices["expected_matrix"]), 1e-5)


def test_oracle_vector_mass_golden(golden_matrices):
    M = _Mesh(golden_matrices)
    mat = seq.Mat(seq.Sparsity((M.evn, M.evn)))
    seq.par_loop(M.K["mass_vector_ffc"], M.elements(3, 3), mat((M.evn[seq.i[0]], M.evn[seq.i[1]]), seq.INC),
                 M.coords(M.evn, seq.READ))
    assert_allclose(mat.values, np.asarray(golden_matrices["expected_vector_matrix"]), 1e-6)


@pytest.mark.parametrize("kernel,itspace,eps", [("rhs", False, 1e-12), ("rhs_ffc", False, 1e-6),
                                                ("rhs_ffc_itspace", True, 1e-6)])
def test_oracle_rhs_golden(golden_matrices, kernel, itspace, eps):
    M = _Mesh(golden_matrices)
    b = seq.Dat(M.nodes, np.zeros(4))
    if itspace:
        seq.par_loop(M.K[kernel], M.elements(3), b(M.en[seq.i[0]], seq.INC), M.coords(M.evn, seq.READ),
                     M.f(M.en, seq.READ))
    else:
        seq.par_loop(M.K[kernel], M.elements, b(M.en, seq.INC), M.coords(M.evn, seq.READ), M.f(M.en, seq.READ))
    assert_allclose(b.data, np.asarray(golden_matrices["expected_rhs"]), eps)


@pytest.mark.parametrize("kernel,itspace", [("rhs_ffc_vector", False), ("rhs_ffc_vector_itspace", True)])
def test_oracle_vec_rhs_golden(golden_matrices, kernel, itspace):
    M = _Mesh(golden_matrices)
    b = seq.Dat(M.vnodes, np.zeros(8))
    if itspace:
        seq.par_loop(M.K[kernel], M.elements(3), b(M.evn[seq.i[0]], seq.INC), M.coords(M.evn, seq.READ),
                     M.f_vec(M.evn, seq.READ))
    else:
        seq.par_loop(M.K[kernel], M.elements, b(M.evn, seq.INC), M.coords(M.evn, seq.READ),
                     M.f_vec(M.evn, seq.READ))
    assert_allclose(b.data, np.asarray(golden_matrices["expected_vec_rhs"]), 1e-6)


def test_oracle_set_and_zero_rows(golden_matrices):
    M = _Mesh(golden_matrices)
    mat = seq.Mat(seq.Sparsity((M.en, M.en)))
    g = seq.Global(1, 1.0, np.float64)
    seq.par_loop(M.K["kernel_inc"], M.elements(3, 3), mat((M.en[seq.i[0]], M.en[seq.i[1]]), seq.INC), g(seq.READ))
    assert mat.array.sum() == 18
    seq.par_loop(M.K["kernel_set"], M.elements(3, 3), mat((M.en[seq.i[0]], M.en[seq.i[1]]), seq.WRITE), g(seq.READ))
    assert_allclose(mat.array, 1.0)
    mat.zero()
    seq.par_loop(M.K["mass"], M.elements(3, 3), mat((M.en[seq.i[0]], M.en[seq.i[1]]), seq.INC),
                 M.coords(M.evn, seq.READ))
    expected = np.asarray(golden_matrices["expected_matrix"])
    expected[0] = [12.0, 0, 0, 0]
    mat.zero_rows([0], 12.0)
    assert_allclose(mat.values, expected, 1e-5)


def _p1_mass(n):
    from test_gpu_parity import P1_MASS, P1_RHS  # the workload kernels
    coords, elem = meshes.square_p1(n)
    nodes, vnodes, els = seq.Set(len(coords)), seq.Set(len(coords), 2), seq.Set(len(elem))
    en, evn = seq.Map(els, nodes, 3, elem), seq.Map(els, vnodes, 3, elem)
    mat = seq.Mat(seq.Sparsity((en, en)))
    x = seq.Dat(vnodes, coords)
    f = seq.Dat(nodes, 2 * coords[:, 0] + 4 * coords[:, 1])
    b = seq.Dat(nodes, np.zeros(len(coords)))
    seq.par_loop(seq.Kernel(P1_MASS, "p1_mass"), els(3, 3), mat((en[seq.i[0]], en[seq.i[1]]), seq.INC),
                 x(evn, seq.READ))
    seq.par_loop(seq.Kernel(P1_RHS, "p1_rhs"), els(3), b(en[seq.i[0]], seq.INC), x(evn, seq.READ),
                 f(en, seq.READ))
    return mat, b


def test_oracle_regression_mass2d_summary():
    """Numbering-invariant match with mass2d_triangle.expected (100x100)."""
    z = np.load(os.path.join(GOLDEN, "mass2d_triangle_summary.npz"))
    mat, b = _p1_mass(100)
    golden = np.sort(np.repeat(z["mat_values"], z["mat_counts"]))
    assert mat.array.size == int(z["nnz"])
    assert np.abs(np.sort(mat.array) - golden).max() < 1e-12 * golden.max()
    assert abs(mat.array.sum() - float(z["mat_sum"])) < 1e-12
    assert abs(b.data.sum() - float(z["b_sum"])) < 1e-12


def test_oracle_plan_coloring_valid():
    """test_coloring.py:84-114 predicate on the restated plan."""
    rng = np.random.default_rng(1)
    el, nd = seq.Set(12), seq.Set(36)
    vals = rng.integers(0, 4, size=(12, 3))
    m = seq.Map(el, nd, 3, vals)
    mat = seq.Mat(seq.Sparsity((m, m)))
    x = seq.Dat(nd, np.zeros(36, np.uint32), np.uint32)
    p = oplan.plan(el, [mat((m[seq.i[0]], m[seq.i[1]]), seq.INC), x(m[0], seq.WRITE)],
                   partition_size=6, matrix_coloring=True)
    assert p.nblocks == 2
    for b in range(p.nblocks):
        for c in range(p.nthrcol[b]):
            counter = np.zeros(36, np.uint32)
            for e in range(b * 6, b * 6 + p.nelems[b]):
                if p.thrcol[e] == c:
                    counter[vals[e][0]] += 1
            assert (counter < 2).all()


def test_oracle_openmp_matches_sequential():
    from pyop2_b200.workloads import airfoil
    grid = meshes.airfoil_grid(30, 15, 2)
    A = airfoil.build(seq, 30, 15, 2, grid=grid)
    seq._CONSTS.clear()
    B = airfoil.build(seq, 30, 15, 2, grid=grid)
    for _ in range(2):
        ra = airfoil.iteration(seq, A)
    # the same chain with the restated OpenMP backend
    orig = seq.par_loop

    def omp_loop(*a, **k):
        return orig(*a, openmp=True, part_size=64, **k)
    try:
        seq.par_loop = omp_loop
        for _ in range(2):
            rb = airfoil.iteration(seq, B)
    finally:
        seq.par_loop = orig
    assert np.abs(A.p_q.data - B.p_q.data).max() <= 1e-12 * np.abs(A.p_q.data).max()
    assert abs(ra.data[0] - rb.data[0]) <= 1e-12 * abs(ra.data[0])


def test_reference_airfoil_kernel_strings_match_restated_kernels():
    """The reference demo's airfoil kernels (tests/golden/airfoil_kernels.json,
    from demo/airfoil_kernels.py) and this package's restated airfoil kernels
    compute the same chain: three outer iterations on the oracle agree to
    1e-13 (they differ only in operation order and float-literal spelling)."""
    import json
    from conftest import rel_err
    from pyop2_b200.workloads import airfoil
    with open(os.path.join(GOLDEN, "airfoil_kernels.json")) as f:
        code = json.load(f)["kernels"]
    seq._CONSTS.clear()
    grid = meshes.airfoil_grid(40, 20, 5)
    A = airfoil.build(seq, 40, 20, 5, grid=grid)
    B = airfoil.build(seq, 40, 20, 5, grid=grid, consts=False)
    B.k_save = seq.Kernel(code["save_soln"], "save_soln")
    B.k_adt = seq.Kernel(code["adt_calc"], "adt_calc")
    B.k_res = seq.Kernel(code["res_calc"], "res_calc")
    B.k_bres = seq.Kernel(code["bres_calc"], "bres_calc")
    B.k_update = seq.Kernel(code["update"], "update")
    for _ in range(3):
        ra = airfoil.iteration(seq, A)
        rb = airfoil.iteration(seq, B)
    assert rel_err(B.p_q.data, A.p_q.data) < 1e-13
    assert rel_err(rb.data, ra.data) < 1e-13
    seq._CONSTS.clear()
