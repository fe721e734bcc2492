"""op2b_mat_zero_rows_static: the Mat row-zeroing entry point that allocates
no device memory, for callers whose device memory is owned by their host
framework (a solver loop applying boundary conditions every time step in a
process that reserved the GPU's memory up front).  Its row list goes through
a fixed scratch array compiled into the library instead of a per-call
allocation.

The test drives it through the C-ABI and checks it against
op2b_mat_zero_rows (which allocates) on the same CSR values, on two calls in
a row with different row lists: the second call must not see anything left
over in the shared scratch by the first.  Both entry points only write
existing values (0 or the diagonal value), so the results must be equal
bit for bit.

This file is collected last, so a run that stops at the first failure has
run every other test before it; it also passes alone in a fresh process."""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def op2(backend):
    from pyop2_b200 import op2 as _op2
    return _op2


def _pattern(op2):
    """A CSR pattern on the device: P1 triangles of a 40 x 40 square."""
    from pyop2_b200.workloads import meshes
    coords, elem = meshes.square_p1(40)
    nodes, els = op2.Set(len(coords)), op2.Set(len(elem))
    m = op2.Map(els, nodes, 3, elem, "elem_node_zz")
    return op2.Sparsity((m, m)), len(coords)


def _values(sp, seed):
    return np.random.default_rng(seed).standard_normal(sp.nz)


def _run(lib, name, buf, sp, rows, diag, elem_bytes=8):
    rows = np.ascontiguousarray(rows, dtype=np.int32)
    rc = getattr(lib, name)(buf.ptr, sp._d_rowptr, sp._d_colidx, sp._lsize,
                            rows.ctypes.data_as(C.POINTER(C.c_int32)), rows.size, float(diag),
                            elem_bytes, 0)
    return rc


def _pool():
    """The device's default stream-ordered memory pool, which the library's
    allocating entry points draw from (cudaMallocAsync)."""
    from cuda.bindings import runtime as rt
    err, pool = rt.cudaDeviceGetDefaultMemPool(0)
    assert err == rt.cudaError_t.cudaSuccess
    return rt, pool


def _pool_attr(rt, pool, attr):
    err, v = rt.cudaMemPoolGetAttribute(pool, attr)
    assert err == rt.cudaError_t.cudaSuccess
    return int(v)


def test_zero_rows_static_matches_allocating_entry_point(op2):
    from pyop2_b200 import _lib, b200
    lib = _lib._lib
    sp, nrows = _pattern(op2)
    rng = np.random.default_rng(1)
    calls = [(rng.choice(nrows, size=700, replace=False), 3.5),
             (rng.choice(nrows, size=11, replace=False), -2.0)]
    for k, (rows, diag) in enumerate(calls):
        vals = _values(sp, 10 + k)
        a = b200.DeviceBuffer(vals.nbytes)
        b = b200.DeviceBuffer(vals.nbytes)
        a.from_host(vals)
        b.from_host(vals)
        assert _run(lib, "op2b_mat_zero_rows", a, sp, rows, diag) == 0, _lib.last_error()
        assert _run(lib, "op2b_mat_zero_rows_static", b, sp, rows, diag) == 0, _lib.last_error()
        ra = np.empty_like(vals)
        rb = np.empty_like(vals)
        a.to_host(ra)
        b.to_host(rb)
        np.testing.assert_array_equal(ra, rb)
        # and the rows really were zeroed around the diagonal
        rp, ci = sp._rowptr, sp._colidx
        r = int(rows[0])
        seg = slice(rp[r], rp[r + 1])
        assert (rb[seg][ci[seg] != r] == 0).all() and (rb[seg][ci[seg] == r] == diag).all()
        untouched = np.ones(nrows, bool)
        untouched[rows] = False
        keep = np.repeat(untouched, np.diff(rp))
        np.testing.assert_array_equal(rb[keep], vals[keep])


def test_zero_rows_static_rejects_oversized_lists(op2):
    from pyop2_b200 import _lib, b200
    lib = _lib._lib
    sp, nrows = _pattern(op2)
    vals = _values(sp, 3)
    buf = b200.DeviceBuffer(vals.nbytes)
    buf.from_host(vals)
    too_many = np.zeros(65536 + 1, dtype=np.int32)
    assert _run(lib, "op2b_mat_zero_rows_static", buf, sp, too_many, 1.0) != 0
    assert "65536" in _lib.last_error()
    # rows outside the matrix and unsupported element sizes are rejected on
    # the host, before anything is copied or launched
    assert _run(lib, "op2b_mat_zero_rows_static", buf, sp, [0, nrows], 1.0) != 0
    assert "outside" in _lib.last_error()
    assert _run(lib, "op2b_mat_zero_rows_static", buf, sp, [-5], 1.0) != 0
    assert _run(lib, "op2b_mat_zero_rows_static", buf, sp, [0], 1.0, elem_bytes=2) != 0
    assert "elem_bytes" in _lib.last_error()
    out = np.empty_like(vals)
    buf.to_host(out)
    np.testing.assert_array_equal(out, vals)


def test_zero_rows_static_allocates_nothing(op2):
    """Calls of the allocation-free entry point take nothing from the
    stream-ordered pool: its high-water mark, reset before the calls, stays at
    or below the memory in use before them.  The allocating entry point, run
    the same way, does raise it (so the probe sees allocations)."""
    import torch
    from cuda.bindings.driver import cuuint64_t
    from pyop2_b200 import _lib, b200
    lib = _lib._lib
    rt, pool = _pool()
    used = rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent
    high = rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh
    sp, nrows = _pattern(op2)
    vals = _values(sp, 4)
    buf = b200.DeviceBuffer(vals.nbytes)
    buf.from_host(vals)
    rows = np.arange(0, nrows, 3)
    assert _run(lib, "op2b_mat_zero_rows_static", buf, sp, rows, 1.0) == 0, _lib.last_error()
    torch.cuda.synchronize()

    def peak_over(name):
        in_use = _pool_attr(rt, pool, used)
        err, = rt.cudaMemPoolSetAttribute(pool, high, cuuint64_t(0))
        assert err == rt.cudaError_t.cudaSuccess
        for diag in (2.0, 3.0, 4.0):
            assert _run(lib, name, buf, sp, rows, diag) == 0, _lib.last_error()
        torch.cuda.synchronize()
        return _pool_attr(rt, pool, high) - in_use

    assert peak_over("op2b_mat_zero_rows_static") <= 0
    assert peak_over("op2b_mat_zero_rows") > 0
