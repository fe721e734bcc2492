"""Overlapped CUDA-graph capture (pyop2_b200/overlap.py, b200.capture): a
captured airfoil iteration whose independent loops run side by side gives
the results of the loops run one after the other in program order (the
reference's execution order, pyop2/cuda.py:656-658), within the rounding
of the atomic adds both orders leave unordered; device work between loops
inside the capture keeps its place."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def op2(backend):
    from pyop2_b200 import op2 as _op2
    return _op2


def _upload(*dats):
    for d in dats:
        d._to_device()


def test_overlapped_airfoil_iteration_matches_program_order(op2):
    from pyop2_b200 import b200, base
    from pyop2_b200 import configuration as cfg
    from pyop2_b200.workloads import airfoil
    cfg.configure(staged_min_size=0)          # res_calc staged, bres_calc atomic
    for c in list(base.Const._defs):
        c.remove_from_namespace()
    A = airfoil.build(op2, 60, 30, 0)
    q0 = A.p_q.data_ro.copy()
    rms = op2.Global(1, 0.0, np.float64, "rms")
    dats = (A.p_q, A.p_qold, A.p_adt, A.p_res)

    def reset():
        A.p_q.data[:] = q0
        A.p_qold.data[:] = q0
        A.p_adt.data[:] = 0.0
        A.p_res.data[:] = 0.0
        _upload(*dats)

    def step():
        rms.zero()
        airfoil.iteration(op2, A, rms)

    reset()
    step()                                    # bind every loop
    out = {}
    for mode in ("program order", "chain graph", "overlapped graph"):
        reset()
        if mode == "program order":
            for _ in range(4):
                step()
        else:
            with b200.capture(overlap=(mode == "overlapped graph")) as g:
                step()
            for _ in range(4):
                g.launch()
            if mode == "overlapped graph":
                segs = g.segments
        out[mode] = (A.p_q.data_ro.copy(), float(rms.data[0]), A.p_res.data_ro.copy())
    ref_q, ref_rms, _ = out["program order"]
    for mode in ("chain graph", "overlapped graph"):
        q, r, _ = out[mode]
        assert np.abs(q - ref_q).max() <= 1e-12 * np.abs(ref_q).max(), mode
        assert abs(r - ref_rms) <= 1e-12 * abs(ref_rms), mode
    # the memset of rms, then 9 loops of one launch each
    loops = [d for is_loop, d in segs if is_loop]
    assert len(segs) == 10 and len(loops) == 9
    assert segs[2][1] == [0]                  # adt_calc does not wait for save_soln
    assert 3 not in segs[4][1]                # bres_calc does not wait for res_calc
    assert segs[5][1] == [0, 1, 2, 3, 4]      # update waits for all of them


def test_overlapped_capture_keeps_other_device_work_in_order(op2):
    """A memset between two loops of the captured block is a barrier: the
    loop after it sees the zeroed Dat even though the two loops touch
    different Dats otherwise."""
    from pyop2_b200 import b200
    n = 1 << 16
    s = op2.Set(n, 1, "s")
    a = op2.Dat(s, np.arange(n, dtype=np.float64), np.float64, "a")
    b = op2.Dat(s, np.zeros(n), np.float64, "b")
    c = op2.Dat(s, np.zeros(n), np.float64, "c")
    k_copy = op2.Kernel("void cp(double *x, double *y) { y[0] = x[0] + 1.0; }", "cp")
    k_acc = op2.Kernel("void acc(double *y, double *z) { z[0] += y[0]; }", "acc")

    def body():
        op2.par_loop(k_copy, s, a(op2.IdentityMap, op2.READ), b(op2.IdentityMap, op2.WRITE))
        b.zero()
        op2.par_loop(k_acc, s, b(op2.IdentityMap, op2.READ), c(op2.IdentityMap, op2.RW))

    body()
    c.zero()
    with b200.capture(overlap=True) as g:
        body()
    for _ in range(3):
        g.launch()
    np.testing.assert_array_equal(c.data_ro.ravel(), np.zeros(n))
    np.testing.assert_array_equal(b.data_ro.ravel(), np.zeros(n))
    assert [is_loop for is_loop, _ in g.segments] == [True, False, True]
    assert g.segments[2][1] == [1]


def test_small_loops_float_beside_big_ones(op2):
    """overlap='small': on a mesh whose cells and edges fill the GPU only
    bres_calc (900 boundary edges) is relaxed -- it runs beside res_calc --
    while the big loops keep program order; results as in program order."""
    from pyop2_b200 import b200, base
    from pyop2_b200.workloads import airfoil
    for c in list(base.Const._defs):
        c.remove_from_namespace()
    A = airfoil.build(op2, 300, 150, 0)
    q0 = A.p_q.data_ro.copy()
    rms = op2.Global(1, 0.0, np.float64, "rms")
    dats = (A.p_q, A.p_qold, A.p_adt, A.p_res)

    def reset():
        A.p_q.data[:] = q0
        A.p_qold.data[:] = q0
        A.p_adt.data[:] = 0.0
        A.p_res.data[:] = 0.0
        _upload(*dats)

    def step():
        rms.zero()
        airfoil.iteration(op2, A, rms)

    reset()
    step()
    reset()
    for _ in range(3):
        step()
    ref_q, ref_rms = A.p_q.data_ro.copy(), float(rms.data[0])
    reset()
    with b200.capture(overlap="small") as g:
        step()
    for _ in range(3):
        g.launch()
    q, r = A.p_q.data_ro.copy(), float(rms.data[0])
    assert np.abs(q - ref_q).max() <= 1e-12 * np.abs(ref_q).max()
    assert abs(r - ref_rms) <= 1e-12 * abs(ref_rms)
    segs = g.segments
    assert len(segs) == 10
    assert 1 in segs[2][1]                    # adt_calc after save_soln (both big)
    assert 2 in segs[3][1]                    # res_calc after adt_calc
    assert 3 not in segs[4][1]                # bres_calc beside res_calc
    assert {3, 4} <= set(segs[5][1])          # update after both
    with pytest.raises(ValueError):
        b200.capture(overlap="sometimes")
    g.close()
