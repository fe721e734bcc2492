"""Test infrastructure: CPU restatement of the linear solve the B200 backend
runs on the device (pyop2_b200.b200.Solver / op2b_cg_solve), used only by
tests and the bench's CPU leg as the checker.

The reference solves with PETSc KSP, defaults 'cg' + 'jacobi'
(pyop2/base.py:1591-1601, pyop2/petsc_base.py:160-220).  PETSc is not
available, so this is the textbook preconditioned conjugate-gradient
iteration (Hestenes and Stiefel) with left Jacobi preconditioning, from
x = 0, with PETSc's default test on the preconditioned residual norm:
converged when ||z_k|| <= max(rtol ||z_0||, atol), diverged when
||z_k|| >= dtol ||z_0||.  Parity is pinned by the reference's own solve
tests (test/unit/test_matrices.py:647-650, 780-783: x equals the field the
RHS was built from) and by numpy's dense solve on small systems.
"""

import numpy as np


def csr_matvec(rowptr, colidx, vals, x):
    """y = A x for a CSR matrix (numpy; rows summed left to right)."""
    rowptr = np.asarray(rowptr)
    prod = np.asarray(vals) * np.asarray(x)[np.asarray(colidx)]
    y = np.zeros(len(rowptr) - 1)
    nz = np.diff(rowptr) > 0
    y[nz] = np.add.reduceat(prod, rowptr[:-1][nz]) if prod.size else 0.0
    return y


def jacobi_inverse(rowptr, colidx, vals):
    n = len(rowptr) - 1
    d = np.zeros(n)
    for r in range(n):
        seg = slice(rowptr[r], rowptr[r + 1])
        hit = np.nonzero(np.asarray(colidx[seg]) == r)[0]
        if hit.size:
            d[r] = vals[rowptr[r] + hit[-1]]
    return np.where(d != 0.0, 1.0 / np.where(d != 0.0, d, 1.0), 1.0)


def cg(rowptr, colidx, vals, b, jacobi=True, rtol=1e-7, atol=1e-50, dtol=1e4, max_it=1000):
    """Returns (x, iterations, reason, residual history); reason 1
    converged, 2 diverged, 3 breakdown, 4 iteration limit."""
    b = np.asarray(b, dtype=np.float64).ravel()
    dinv = jacobi_inverse(rowptr, colidx, vals) if jacobi else np.ones_like(b)
    x = np.zeros_like(b)
    r = b.copy()
    z = dinv * r
    p = z.copy()
    rz = r @ z
    r0 = np.sqrt(z @ z)
    hist = [r0]
    ttol = max(rtol * r0, atol)
    if r0 <= ttol:
        return x, 0, 1, hist
    if not np.isfinite(r0):
        return x, 0, 3, hist
    for k in range(max_it):
        q = csr_matvec(rowptr, colidx, vals, p)
        pq = p @ q
        alpha = rz / pq if (pq != 0.0 and np.isfinite(pq)) else 0.0
        x += alpha * p
        r -= alpha * q
        z = dinv * r
        rz_new = r @ z
        beta = rz_new / rz if (rz != 0.0 and np.isfinite(rz)) else 0.0
        p = z + beta * p
        rz = rz_new
        rn = np.sqrt(z @ z)
        hist.append(rn)
        if not np.isfinite(rn):
            return x, k + 1, 3, hist
        if rn <= ttol:
            return x, k + 1, 1, hist
        if rn >= dtol * r0:
            return x, k + 1, 2, hist
    return x, max_it, 4, hist
