"""The CPU restatement of the linear solve (oracle/linalg.py) against numpy's
dense algebra: the checker of the device solve is itself checked here."""

import numpy as np

from oracle import linalg, seq
from pyop2_b200.workloads import fem, meshes


def _p1_mass(n):
    coords, elem = meshes.square_p1(n)
    P = fem.build_p1(seq, n, coords=coords, elem=elem)
    fem.assemble_p1(seq, P)
    return P.sparsity.rowptr, P.sparsity.colidx, P.mat.array, P.mat.values


def test_matvec_and_cg_match_dense_solve():
    rp, ci, vals, dense = _p1_mass(12)
    rng = np.random.default_rng(0)
    f = rng.standard_normal(dense.shape[0])
    np.testing.assert_allclose(linalg.csr_matvec(rp, ci, vals, f), dense @ f, rtol=1e-13, atol=1e-16)
    b = dense @ f
    for jacobi in (True, False):
        x, its, reason, hist = linalg.cg(rp, ci, vals, b, jacobi=jacobi, rtol=1e-12)
        assert reason == 1 and 0 < its < 200 and len(hist) == its + 1
        assert np.abs(x - np.linalg.solve(dense, b)).max() < 1e-8 * np.abs(f).max()


def test_cg_reasons():
    rp, ci, vals, dense = _p1_mass(8)
    b = dense @ np.random.default_rng(1).standard_normal(dense.shape[0])
    x, its, reason, hist = linalg.cg(rp, ci, vals, b, max_it=2, rtol=1e-14)
    assert (its, reason) == (2, 4)
    x, its, reason, hist = linalg.cg(rp, ci, vals, np.zeros_like(b))
    assert (its, reason) == (0, 1) and not x.any()
