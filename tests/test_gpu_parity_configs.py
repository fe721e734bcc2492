"""Parity at the benchmark configurations' own sizes: the B200 backend
against the CPU oracle (the reference's sequential backend restated,
pyop2/sequential.py:55-121 with the argument expressions of
pyop2/host.py:91-207) on the same seeded inputs.

* P1 mass + RHS on the 256 x 256 unit square (131,072 triangles, 66,049
  nodes): Sparsity bit-exact with nnz = 460,289; Mat and RHS within 1e-12.
* Airfoil chain on the permuted 1200 x 600 mesh (720,000 cells, 1,438,200
  edges): each loop once in the default forms (direct loops bit-exact,
  indirect INC within 1e-12), then three more outer iterations: q and rms
  within 1e-12.
* P2 stiffness + mass on the jittered 1024 x 1024 grid (2,097,152 triangles,
  4,198,401 dofs, nnz 48,250,881): Sparsity bit-exact, FP64 Mats within
  1e-12; the precision form (FP32 element math, FP64 Kahan-compensated
  two-phase accumulation) within 1e-5 of the FP64 oracle, the error stated
  per Mat.
* Batching: 4096 uneven P1 meshes (elements log-uniform in [2^8, 2^16]) in
  tuned batched launches; a sample of meshes (smallest, largest, and some in
  between) against the oracle within 1e-12.
* Serving: airfoil chain requests (10 iterations) and P1 assembly requests
  served by the continuous-batching engine in one mix, each against the
  oracle run on the same mesh and request parameter, within 1e-12.

Tolerance: max|gpu - cpu| / max|cpu| (normwise relative), in FP64; INC order
differs from element order on the GPU (staged colour rounds, atomics), so
bit equality is not expected there.
"""

import numpy as np
import pytest

from conftest import rel_err
from oracle import seq
from pyop2_b200.workloads import airfoil, fem, meshes

pytestmark = pytest.mark.gpu
TOL = 1e-12
TOL_PRECISION_FORM = 1e-5


@pytest.fixture
def op2(backend):
    from pyop2_b200 import op2 as _op2
    _clear_consts()
    yield _op2
    _clear_consts()


def _clear_consts():
    from pyop2_b200 import base
    for c in list(base.Const._defs):
        c.remove_from_namespace()
    seq._CONSTS.clear()


def test_p1_256_mass_rhs_matches_oracle(op2):
    G, O = fem.build_p1(op2, 256), fem.build_p1(seq, 256)
    assert G.n_elem == 131072 and G.n_nodes == 66049
    fem.assemble_p1(op2, G)
    fem.assemble_p1(seq, O)
    assert O.sparsity.nz == 460289
    np.testing.assert_array_equal(G.sparsity._rowptr, O.sparsity.rowptr)
    np.testing.assert_array_equal(G.sparsity._colidx, O.sparsity.colidx)
    assert rel_err(G.mat.array, O.mat.array) < TOL
    assert rel_err(G.b.data_ro, O.b.data) < TOL


def test_airfoil_1200x600_matches_oracle(op2):
    from pyop2_b200 import b200
    grid = meshes.airfoil_grid(1200, 600, 0)
    assert (grid.ncells, grid.nedges, grid.nbedges) == (720000, 1438200, 3600)
    G = airfoil.build(op2, 1200, 600, 0, grid=grid)
    O = airfoil.build(seq, 1200, 600, 0, grid=grid)
    airfoil.save_soln(op2, G)
    airfoil.save_soln(seq, O)
    np.testing.assert_array_equal(G.p_qold.data_ro, O.p_qold.data)
    airfoil.adt_calc(op2, G)
    airfoil.adt_calc(seq, O)
    np.testing.assert_array_equal(G.p_adt.data_ro, O.p_adt.data)
    airfoil.res_calc(op2, G)
    airfoil.res_calc(seq, O)
    assert rel_err(G.p_res.data_ro, O.p_res.data) < TOL
    # res_calc ran in the backend's default form for this size
    modes = {bl.spec.mode for bl in b200.ParLoop._bound_cache.values()
             if bl.spec.kernel_name == "res_calc"}
    assert "staged" in modes
    airfoil.bres_calc(op2, G)
    airfoil.bres_calc(seq, O)
    assert rel_err(G.p_res.data_ro, O.p_res.data) < TOL
    g_rms = op2.Global(1, 0.0, np.float64, "rms")
    o_rms = seq.Global(1, 0.0, np.float64, "rms")
    airfoil.update(op2, G, g_rms)
    airfoil.update(seq, O, o_rms)
    assert rel_err(G.p_q.data_ro, O.p_q.data) < TOL
    assert rel_err(G.p_res.data_ro, O.p_res.data) < TOL
    assert rel_err(g_rms.data, o_rms.data) < TOL
    for _ in range(3):
        gr = airfoil.iteration(op2, G)
        orr = airfoil.iteration(seq, O)
        assert rel_err(gr.data, orr.data) < TOL
    assert rel_err(G.p_q.data_ro, O.p_q.data) < TOL


@pytest.fixture(scope="module")
def p2_oracle():
    """The FP64 sequential oracle's P2 1024 x 1024 stiffness and mass."""
    O = fem.build_p2(seq, 1024, seed=0)
    fem.assemble_p2(seq, O)
    return O


@pytest.mark.parametrize("form", ["f64", "f64_lma", "f32_lma_kahan"])
def test_p2_1024_matches_oracle(op2, p2_oracle, form):
    """FP64 in the default (atomic) and the two-phase form within 1e-12;
    the precision form within 1e-5 per Mat (its FP32 element math sets the
    error; the FP64 Kahan-compensated accumulation adds nothing visible)."""
    from pyop2_b200 import configuration as cfg
    prec, mode, kahan = {"f64": ("f64", None, False), "f64_lma": ("f64", "lma", False),
                         "f32_lma_kahan": ("f32", "lma", True)}[form]
    if mode:
        cfg.configure(inc_mode=mode, kahan=kahan)
    O = p2_oracle
    G = fem.build_p2(op2, 1024, seed=0, precision=prec)
    assert G.n_elem == 2097152 and G.n_dofs == 4198401
    fem.assemble_p2(op2, G)
    assert G.sparsity.nz == 48250881
    if form == "f64":
        np.testing.assert_array_equal(G.sparsity._rowptr, O.sparsity.rowptr)
        np.testing.assert_array_equal(G.sparsity._colidx, O.sparsity.colidx)
    tol = TOL if prec == "f64" else TOL_PRECISION_FORM
    e_k = rel_err(G.K.array, O.K.array)
    e_m = rel_err(G.M.array, O.M.array)
    print("P2 1024 %s: max rel err K %.3e M %.3e" % (form, e_k, e_m))
    assert e_k < tol and e_m < tol


def test_batched_meshes_match_oracle(op2):
    """The batching configuration (4096 meshes) in tuned batched launches;
    sample meshes against the oracle."""
    from pyop2_b200 import autotune, b200
    from pyop2_b200.batch import BatchLoop
    from pyop2_b200.workloads import batching
    shapes = batching.mesh_shapes(4096, 0)
    probs = batching.build(op2, shapes, 0)
    loops = [autotune.tuned_batch(insts, reps=1) for insts in batching.instances(op2, probs)]
    for P in probs:
        P.mat.zero()
        P.stiff.zero()
        P.b.zero()
    for bl in loops:
        bl.launch()
    b200.synchronize()
    sizes = [P.n_elem for P in probs]
    sample = sorted({0, 1, 1000, 2048, 4095, int(np.argmin(sizes)), int(np.argmax(sizes))})
    for i in sample:
        P = probs[i]
        Q = fem.build_p1(seq, 0, coords=P.coords.data_ro, elem=P.elem_node.values, stiffness=True)
        fem.assemble_p1(seq, Q)
        fem.assemble_p1_stiffness(seq, Q)
        np.testing.assert_array_equal(P.sparsity._rowptr, Q.sparsity.rowptr)
        np.testing.assert_array_equal(P.sparsity._colidx, Q.sparsity.colidx)
        assert rel_err(P.mat.array, Q.mat.array) < TOL, i
        assert rel_err(P.stiff.array, Q.stiff.array) < TOL, i
        assert rel_err(P.b.data_ro, Q.b.data) < TOL, i
    assert all(isinstance(bl, BatchLoop) for bl in loops)


def _oracle_chain(grid, scale, iters):
    """An airfoil chain request on the oracle: q = qinf + s (q_base - qinf),
    save_soln, then ``iters`` x (adt_calc, res_calc, bres_calc, update) with
    one rms Global summed over all updates (pyop2_b200.serve.ChainJob)."""
    from pyop2_b200 import serve
    O = airfoil.build(seq, 0, 0, grid=grid, consts=False)
    q_base = seq.Dat(O.vcells, airfoil.initial_q(grid.ncells, 1), np.float64, "q_base")
    s = seq.Global(1, scale, np.float64, "s")
    O.p_res.data[...] = 0.0
    seq.par_loop(seq.Kernel(serve.Q_INIT, "q_init"), O.cells, O.p_q(seq.IdentityMap, seq.WRITE),
                 q_base(seq.IdentityMap, seq.READ), s(seq.READ))
    airfoil.save_soln(seq, O)
    rms = seq.Global(1, 0.0, np.float64, "rms")
    for _ in range(iters):
        airfoil.adt_calc(seq, O)
        airfoil.res_calc(seq, O)
        airfoil.bres_calc(seq, O)
        airfoil.update(seq, O, rms)
    return O.p_q.data, rms.data


def test_served_requests_match_oracle(op2):
    """Chain and assembly requests served in one mix by the engine, each
    against the oracle."""
    from pyop2_b200 import serve
    from pyop2_b200.workloads import serving
    consts = serving.declare_consts(op2)
    oconsts = serving.declare_consts(seq)
    pool = serving.mesh_pool(3, 3, seed=21, p1_range=(1e3, 1e5), quad_range=(1e4, 1e5))
    store = serve.MeshStore(budget=20 << 30)
    serving.register(store, op2, pool, seed=21)
    jobs = serving.trace(24, 1e5, pool, seed=9, iters=10)
    eng = serve.Engine(store, consumer=serve.keep_results)
    done = eng.run(serving.clone_trace(jobs, realtime=False), realtime=False)
    assert len(done) == len(jobs) and max(eng.batch_sizes) > 1
    checked = {"quad": 0, "p1": 0}
    for j in done:
        if checked[j.kind] >= 3:
            continue
        mesh = store.get(j.mesh_id)
        scale = serve.request_scale(j.seed)
        if j.kind == "quad":
            q, rms = _oracle_chain(mesh.A.grid, scale, j.iters)
            assert rel_err(j.result["q"], q) < TOL, j.rid
            assert rel_err(j.result["rms"], rms) < TOL, j.rid
        else:
            P = mesh.P
            Q = fem.build_p1(seq, 0, coords=P.coords.data_ro, elem=P.elem_node.values)
            Q.f.data[:] = scale * P.f.data_ro.reshape(Q.f.data.shape)
            fem.assemble_p1(seq, Q)
            assert rel_err(j.result["mat"], Q.mat.array) < TOL, j.rid
            assert rel_err(j.result["b"], Q.b.data.reshape(-1)) < TOL, j.rid
        checked[j.kind] += 1
    assert checked == {"quad": 3, "p1": 3}
    del consts, oconsts


def _reference_kernels(api, A):
    """Swap the chain's kernels for the reference demo's own kernel strings
    (demo/airfoil_kernels.py), unchanged."""
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "airfoil_kernels.json")) as f:
        code = json.load(f)["kernels"]
    A.k_save = api.Kernel(code["save_soln"], "save_soln")
    A.k_adt = api.Kernel(code["adt_calc"], "adt_calc")
    A.k_res = api.Kernel(code["res_calc"], "res_calc")
    A.k_bres = api.Kernel(code["bres_calc"], "bres_calc")
    A.k_update = api.Kernel(code["update"], "update")
    return A


def test_reference_airfoil_kernel_strings_1200x600(op2):
    """The reference user's airfoil kernels, exactly as its demo passes them
    to op2.Kernel (float literals, its own local names), compiled by NVRTC
    into the stubs and run on the 1200 x 600 permuted mesh in the default
    forms, against the oracle running the same strings."""
    grid = meshes.airfoil_grid(1200, 600, 0)
    G = _reference_kernels(op2, airfoil.build(op2, 1200, 600, 0, grid=grid))
    O = _reference_kernels(seq, airfoil.build(seq, 1200, 600, 0, grid=grid))
    airfoil.save_soln(op2, G)
    airfoil.save_soln(seq, O)
    np.testing.assert_array_equal(G.p_qold.data_ro, O.p_qold.data)
    airfoil.adt_calc(op2, G)
    airfoil.adt_calc(seq, O)
    np.testing.assert_array_equal(G.p_adt.data_ro, O.p_adt.data)
    airfoil.res_calc(op2, G)
    airfoil.res_calc(seq, O)
    assert rel_err(G.p_res.data_ro, O.p_res.data) < TOL
    for _ in range(2):
        gr = airfoil.iteration(op2, G)
        orr = airfoil.iteration(seq, O)
        assert rel_err(gr.data, orr.data) < TOL
    assert rel_err(G.p_q.data_ro, O.p_q.data) < TOL
