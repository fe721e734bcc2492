"""Workload parity: the B200 backend against the CPU oracle (the sequential
backend restated) on the same seeded inputs.

Tolerances: direct loops compute in the same IEEE operation order on both
sides (the stubs are compiled without FMA contraction, like the host
compiler's baseline x86-64 code), so they are compared bit for bit.  Loops
that INC into shared nodes or Mat entries sum in a different order (block and
thread colours instead of element order): FP64 results agree within 1e-12
normwise relative error, max|gpu - cpu| / max|cpu|."""

import numpy as np
import pytest

from conftest import rel_err
from oracle import seq
from pyop2_b200.workloads import airfoil, meshes

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture
def op2(backend):
    from pyop2_b200 import op2 as _op2
    return _op2


def _clear_consts(op2mod):
    from pyop2_b200 import base
    for c in list(base.Const._defs):
        c.remove_from_namespace()
    seq._CONSTS.clear()


@pytest.fixture(params=["atomic", "color", "lma", "staged", "gather"])
def inc_mode(request):
    """Run a test under both INC conflict strategies of indirect loops."""
    from pyop2_b200 import configuration as cfg
    old = (cfg.cfg['inc_mode'], cfg.cfg['staged_min_size'])
    cfg.configure(inc_mode=request.param, staged_min_size=0)
    yield request.param
    cfg.configure(inc_mode=old[0], staged_min_size=old[1])


@pytest.mark.parametrize("nx,ny,seed", [(24, 12, 0), (60, 30, 1)])
def test_airfoil_chain_matches_oracle(op2, nx, ny, seed, inc_mode):
    _clear_consts(op2)
    grid = meshes.airfoil_grid(nx, ny, seed)
    G = airfoil.build(op2, nx, ny, seed, grid=grid)
    O = airfoil.build(seq, nx, ny, seed, grid=grid)
    # one loop at a time first: direct loops bit-exact, indirect within TOL
    airfoil.save_soln(op2, G)
    airfoil.save_soln(seq, O)
    np.testing.assert_array_equal(G.p_qold.data_ro, O.p_qold.data)
    airfoil.adt_calc(op2, G)
    airfoil.adt_calc(seq, O)
    np.testing.assert_array_equal(G.p_adt.data_ro, O.p_adt.data)
    airfoil.res_calc(op2, G)
    airfoil.res_calc(seq, O)
    assert rel_err(G.p_res.data_ro, O.p_res.data) < TOL
    airfoil.bres_calc(op2, G)
    airfoil.bres_calc(seq, O)
    assert rel_err(G.p_res.data_ro, O.p_res.data) < TOL
    g_rms = op2.Global(1, 0.0, np.float64, "rms")
    o_rms = seq.Global(1, 0.0, np.float64, "rms")
    airfoil.update(op2, G, g_rms)
    airfoil.update(seq, O, o_rms)
    assert rel_err(G.p_q.data_ro, O.p_q.data) < TOL
    assert rel_err(g_rms.data, o_rms.data) < TOL
    # then full iterations
    for _ in range(3):
        gr = airfoil.iteration(op2, G)
        orr = airfoil.iteration(seq, O)
    assert rel_err(G.p_q.data_ro, O.p_q.data) < 1e-11
    assert rel_err(gr.data, orr.data) < 1e-11
    _clear_consts(op2)


def test_airfoil_results_repeatable(op2):
    """Coloured INC (inc_mode='color'): same inputs, same plan, bit-identical
    results on every run."""
    from pyop2_b200 import configuration as cfg
    old = cfg.cfg['inc_mode']
    cfg.configure(inc_mode='color')
    try:
        _repeatable(op2)
    finally:
        cfg.configure(inc_mode=old)


def _repeatable(op2):
    _clear_consts(op2)
    grid = meshes.airfoil_grid(40, 20, 3)
    outs = []
    for _ in range(2):
        G = airfoil.build(op2, 40, 20, 3, grid=grid, consts=not outs)
        for _ in range(2):
            r = airfoil.iteration(op2, G)
        outs.append((G.p_q.data_ro.copy(), r.data.copy()))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
    _clear_consts(op2)


P1_MASS = """
void p1_mass(double A[1][1], double *x[2], int j, int k) {
  double a00 = x[1][0] - x[0][0], a01 = x[2][0] - x[0][0];
  double a10 = x[1][1] - x[0][1], a11 = x[2][1] - x[0][1];
  double area = fabs(a00 * a11 - a01 * a10);
  const double w = 1.0 / 6.0;
  const double phi[3][3] = {{2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0},
                            {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0},
                            {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0}};
  for (int q = 0; q < 3; q++) A[0][0] += phi[q][j] * phi[q][k] * w * area;
}
"""

P1_RHS = """
void p1_rhs(double *b, double *x[2], double **f, int j) {
  double a00 = x[1][0] - x[0][0], a01 = x[2][0] - x[0][0];
  double a10 = x[1][1] - x[0][1], a11 = x[2][1] - x[0][1];
  double area = fabs(a00 * a11 - a01 * a10);
  const double w = 1.0 / 6.0;
  const double phi[3][3] = {{2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0},
                            {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0},
                            {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0}};
  for (int q = 0; q < 3; q++) {
    double fq = 0.0;
    for (int r = 0; r < 3; r++) fq += phi[q][r] * f[r][0];
    b[0] += phi[q][j] * fq * w * area;
  }
}
"""


def _p1(api, coords, elem, fvals):
    nodes = api.Set(len(coords), 1, "nodes")
    vnodes = api.Set(len(coords), 2, "vnodes")
    els = api.Set(len(elem), 1, "elements")
    en = api.Map(els, nodes, 3, elem, "elem_node")
    evn = api.Map(els, vnodes, 3, elem, "elem_vnode")
    sp = api.Sparsity((en, en), "sp")
    mat = api.Mat(sp, np.float64, "mat")
    x = api.Dat(vnodes, coords, np.float64, "coords")
    f = api.Dat(nodes, fvals, np.float64, "f")
    b = api.Dat(nodes, np.zeros(len(coords)), np.float64, "b")
    api.par_loop(api.Kernel(P1_MASS, "p1_mass"), els(3, 3), mat((en[api.i[0]], en[api.i[1]]), api.INC),
                 x(evn, api.READ))
    api.par_loop(api.Kernel(P1_RHS, "p1_rhs"), els(3), b(en[api.i[0]], api.INC), x(evn, api.READ),
                 f(en, api.READ))
    return mat, b, sp


@pytest.mark.parametrize("n", [16, 100])
def test_p1_mass_rhs_matches_oracle(op2, n, inc_mode):
    coords, elem = meshes.square_p1(n)
    fvals = np.sin(np.pi * coords[:, 0]) * np.sin(np.pi * coords[:, 1])
    gm, gb, gsp = _p1(op2, coords, elem, fvals)
    om, ob, osp = _p1(seq, coords, elem, fvals)
    np.testing.assert_array_equal(gsp._rowptr, osp.rowptr)
    np.testing.assert_array_equal(gsp._colidx, osp.colidx)
    assert rel_err(gm.array, om.array) < TOL
    assert rel_err(gb.data_ro, ob.data) < TOL


@pytest.mark.parametrize("dtype,cdim", [(np.float64, 3), (np.float32, 3), (np.int32, 1)])
def test_staged_edge_cases_match_oracle(op2, dtype, cdim):
    """The staged form on a random edge graph where some edges have both
    ends at one node (a thread adds twice to one staged row), INC rows of
    odd width and of float32 / int32, a direct READ arg (read at the
    reordered element) and a Global MAX, against the sequential oracle."""
    from pyop2_b200 import configuration as cfg
    rng = np.random.default_rng(11)
    nnodes, nedges = 3000, 20000
    e2n = rng.integers(0, nnodes, size=(nedges, 2)).astype(np.int32)
    e2n[::97, 1] = e2n[::97, 0]                       # degenerate edges
    w = rng.integers(1, 5, size=nedges).astype(dtype)
    ctype = {np.float64: "double", np.float32: "float", np.int32: "int"}[dtype]
    code = """void k(%(t)s *a, %(t)s *b, %(t)s *w, %(t)s *g) {
  for (int i = 0; i < %(c)d; ++i) { a[i] += (%(t)s)(i + 1) * w[0]; b[i] += w[0]; }
  if (w[0] > g[0]) g[0] = w[0];
}""" % {"t": ctype, "c": cdim}
    old = (cfg.cfg['inc_mode'], cfg.cfg['staged_min_size'])
    cfg.configure(inc_mode="staged", staged_min_size=0)
    try:
        res = []
        for api in (op2, seq):
            edges, nodes = api.Set(nedges, 1, "edges"), api.Set(nnodes, cdim, "nodes")
            m = api.Map(edges, nodes, 2, e2n, "e2n")
            x = api.Dat(nodes, np.zeros((nnodes, cdim), dtype), dtype, "x")
            wd = api.Dat(edges, w.copy(), dtype, "w")
            g = api.Global(1, 0, dtype, "g")
            api.par_loop(api.Kernel(code, "k"), edges, x(m[0], api.INC), x(m[1], api.INC),
                         wd(api.IdentityMap, api.READ), g(api.MAX))
            res.append((np.array(x.data_ro if api is op2 else x.data), np.array(g.data)))
        from pyop2_b200 import b200
        assert any(bl.spec.mode == "staged" for bl in b200.ParLoop._bound_cache.values()
                   if bl.spec.kernel_name == "k")
        if dtype == np.int32:
            np.testing.assert_array_equal(res[0][0], res[1][0])
        else:
            assert rel_err(res[0][0], res[1][0]) < (1e-12 if dtype == np.float64 else 1e-6)
        np.testing.assert_array_equal(res[0][1], res[1][1])
    finally:
        cfg.configure(inc_mode=old[0], staged_min_size=old[1])


@pytest.mark.parametrize("dtype,cdim", [(np.float64, 4), (np.float64, 8), (np.float64, 16),
                                        (np.float32, 8), (np.int32, 32)])
def test_staged_wide_rows_match_oracle(op2, dtype, cdim):
    """Staged READ rows and INC accumulators of 32, 64 and 128 bytes, whose
    16-byte chunks the staged form keeps in a permuted order in shared
    memory, against the sequential oracle."""
    from pyop2_b200 import configuration as cfg
    rng = np.random.default_rng(5)
    nnodes, nedges = 2000, 15000
    e2n = rng.integers(0, nnodes, size=(nedges, 2)).astype(np.int32)
    e2n[::53, 1] = e2n[::53, 0]
    y0 = rng.integers(-50, 50, size=(nnodes, cdim)).astype(dtype)
    ctype = {np.float64: "double", np.float32: "float", np.int32: "int"}[dtype]
    code = """void kwr(%(t)s *a, %(t)s *b, %(t)s *y0, %(t)s *y1) {
  for (int i = 0; i < %(c)d; ++i) { a[i] += y1[i] * (%(t)s)(i + 1); b[i] += y0[i] - y1[(i + 1) %% %(c)d]; }
}""" % {"t": ctype, "c": cdim}
    old = (cfg.cfg['inc_mode'], cfg.cfg['staged_min_size'])
    cfg.configure(inc_mode="staged", staged_min_size=0)
    try:
        res = []
        for api in (op2, seq):
            edges, nodes = api.Set(nedges, 1, "edges"), api.Set(nnodes, cdim, "nodes")
            m = api.Map(edges, nodes, 2, e2n, "e2n")
            x = api.Dat(nodes, np.zeros((nnodes, cdim), dtype), dtype, "x")
            y = api.Dat(nodes, y0.copy(), dtype, "y")
            api.par_loop(api.Kernel(code, "kwr"), edges, x(m[0], api.INC), x(m[1], api.INC),
                         y(m[0], api.READ), y(m[1], api.READ))
            res.append(np.array(x.data_ro if api is op2 else x.data))
        from pyop2_b200 import b200
        assert any(bl.spec.mode == "staged" for bl in b200.ParLoop._bound_cache.values()
                   if bl.spec.kernel_name == "kwr")
        if dtype == np.int32:
            np.testing.assert_array_equal(res[0], res[1])
        else:
            assert rel_err(res[0], res[1]) < (1e-12 if dtype == np.float64 else 1e-6)
    finally:
        cfg.configure(inc_mode=old[0], staged_min_size=old[1])


def test_staged_too_wide_falls_back_to_atomic(op2):
    """INC rows too wide for the staged form's shared memory (128 doubles
    per row, ~380 distinct targets per block: ~390 KB) run in the atomic
    form, with the oracle's results."""
    from pyop2_b200 import b200
    from pyop2_b200 import configuration as cfg
    rng = np.random.default_rng(12)
    nnodes, nedges, cdim = 20000, 60000, 128
    e2n = rng.integers(0, nnodes, size=(nedges, 2)).astype(np.int32)
    code = """void kw(double *a, double *b) {
  for (int i = 0; i < 128; ++i) { a[i] += 1.0 + i; b[i] += 0.5 * i; }
}"""
    old = (cfg.cfg['inc_mode'], cfg.cfg['staged_min_size'])
    cfg.configure(inc_mode="staged", staged_min_size=0)
    try:
        out = []
        for api in (op2, seq):
            edges, nodes = api.Set(nedges, 1, "edges"), api.Set(nnodes, cdim, "nodes")
            m = api.Map(edges, nodes, 2, e2n, "e2n")
            x = api.Dat(nodes, np.zeros((nnodes, cdim)), np.float64, "x")
            api.par_loop(api.Kernel(code, "kw"), edges, x(m[0], api.INC), x(m[1], api.INC))
            out.append(np.array(x.data_ro if api is op2 else x.data))
        modes = {bl.spec.mode for bl in b200.ParLoop._bound_cache.values() if bl.spec.kernel_name == "kw"}
        assert modes == {"atomic"}
        assert rel_err(out[0], out[1]) < 1e-12
    finally:
        cfg.configure(inc_mode=old[0], staged_min_size=old[1])


def test_owner_mode_is_bit_exact(op2):
    """Owner-computes adds each target's contributions in element order
    starting from its current value -- the sequential backend's order -- so
    the Mat, the RHS and the airfoil residual equal the oracle bit for bit."""
    from pyop2_b200 import configuration as cfg
    old = (cfg.cfg['owner_mode'], cfg.cfg['inc_mode'])
    cfg.configure(owner_mode='always')
    try:
        coords, elem = meshes.square_p1(40)
        fvals = np.sin(np.pi * coords[:, 0]) * np.sin(np.pi * coords[:, 1])
        gm, gb, _ = _p1(op2, coords, elem, fvals)
        om, ob, _ = _p1(seq, coords, elem, fvals)
        np.testing.assert_array_equal(gm.array, om.array)
        # the RHS kernel adds three quadrature terms per call: the sequential
        # backend adds each into the global value, owner-computes sums them in
        # the zeroed local first, so only rounding of those sums differs
        assert rel_err(gb.data_ro, ob.data) < 1e-15
        _clear_consts(op2)
        grid = meshes.airfoil_grid(30, 16, 5)
        G = airfoil.build(op2, 30, 16, 5, grid=grid)
        O = airfoil.build(seq, 30, 16, 5, grid=grid)
        for api, A in ((op2, G), (seq, O)):
            airfoil.save_soln(api, A)
            airfoil.adt_calc(api, A)
            airfoil.res_calc(api, A)
            airfoil.bres_calc(api, A)
        np.testing.assert_array_equal(G.p_res.data_ro, O.p_res.data)
    finally:
        cfg.configure(owner_mode=old[0], inc_mode=old[1])
        _clear_consts(op2)


def test_owner_mode_kahan_matches(op2):
    from pyop2_b200 import configuration as cfg
    cfg.configure(kahan=True, owner_mode='auto')
    try:
        coords, elem = meshes.square_p1(24)
        fvals = coords[:, 0] + 2 * coords[:, 1]
        gm, gb, _ = _p1(op2, coords, elem, fvals)
        om, ob, _ = _p1(seq, coords, elem, fvals)
        assert rel_err(gm.array, om.array) < 1e-15
        assert rel_err(gb.data_ro, ob.data) < 1e-15
    finally:
        cfg.configure(kahan=False, owner_mode='never')


def test_p1_mass_regression_golden(op2):
    """The 100x100 mass problem of the reference's regression test
    (test/regression/tests/mass2d_triangle): the golden's mesh numbering is
    not available, so numbering-invariant quantities are compared: the
    multiset of Mat values and the Mat total (within 1e-12 of each value's
    magnitude), and the RHS total for f = 2x + 4y."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "mass2d_triangle_summary.npz"))
    coords, elem = meshes.square_p1(100)
    fvals = 2 * coords[:, 0] + 4 * coords[:, 1]
    gm, gb, _ = _p1(op2, coords, elem, fvals)
    vals = np.sort(gm.array)
    golden = np.sort(np.repeat(z["mat_values"], z["mat_counts"]))
    assert vals.size == int(z["nnz"])
    assert np.abs(vals - golden).max() < 1e-12 * np.abs(golden).max()
    assert abs(gm.array.sum() - float(z["mat_sum"])) < 1e-12
    assert abs(gb.data_ro.sum() - float(z["b_sum"])) < 1e-12


def test_p1_mass_regression_golden_via_triangle_files(op2, tmp_path):
    """The same regression problem read through the Triangle reader
    (pyop2/demo/mass2d_triangle.py reads its mesh with
    demo/triangle_reader.py): mesh written as .node/.ele, read back into op2
    objects, assembled, compared with the golden's invariants."""
    import os
    from pyop2_b200 import triangle_reader
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "mass2d_triangle_summary.npz"))
    coords, elem = meshes.square_p1(100)
    prefix = str(tmp_path / "square")
    triangle_reader.write_triangle(prefix, coords, elem)
    nodes, vnodes, x, els, en, evn = triangle_reader.read_triangle(prefix, op2)
    f = op2.Dat(nodes, 2 * x.data_ro[:, 0] + 4 * x.data_ro[:, 1], np.float64, "f")
    b = op2.Dat(nodes, np.zeros(nodes.size), np.float64, "b")
    mat = op2.Mat(op2.Sparsity((en, en), "sp"), np.float64, "mat")
    op2.par_loop(op2.Kernel(P1_MASS, "p1_mass"), els(3, 3), mat((en[op2.i[0]], en[op2.i[1]]), op2.INC),
                 x(evn, op2.READ))
    op2.par_loop(op2.Kernel(P1_RHS, "p1_rhs"), els(3), b(en[op2.i[0]], op2.INC), x(evn, op2.READ),
                 f(en, op2.READ))
    vals = np.sort(mat.array)
    golden = np.sort(np.repeat(z["mat_values"], z["mat_counts"]))
    assert vals.size == int(z["nnz"])
    assert np.abs(vals - golden).max() < 1e-12 * np.abs(golden).max()
    assert abs(b.data_ro.sum() - float(z["b_sum"])) < 1e-12


def test_airfoil_from_mesh_file_layout_matches_oracle(op2):
    """The airfoil problem declared from a mesh-file layout through
    fromhdf5 (as pyop2/demo/airfoil.py:45-75 declares it) runs the chain to
    the oracle's results."""
    from test_mesh_io import H5File
    _clear_consts(op2)
    grid = meshes.airfoil_grid(40, 20, 5)
    G = airfoil.build_from_hdf5(op2, H5File.from_layout(airfoil.hdf5_layout(grid, seed=5)))
    O = airfoil.build(seq, 40, 20, 5, grid=grid)
    for _ in range(2):
        gr = airfoil.iteration(op2, G)
        orr = airfoil.iteration(seq, O)
    assert rel_err(G.p_q.data_ro, O.p_q.data) < 1e-11
    assert rel_err(gr.data, orr.data) < 1e-11
    _clear_consts(op2)


def test_two_phase_is_bit_exact_and_launch_independent(op2):
    """inc_mode='lma' adds each target's contributions in element order
    starting from its current value -- the sequential backend's order -- so
    the Mat and the airfoil residual equal the oracle bit for bit, and the
    result does not depend on the block size."""
    from pyop2_b200 import configuration as cfg
    old = (cfg.cfg['inc_mode'], cfg.cfg['block_size'])
    try:
        mats = []
        for bs in (128, 512):
            cfg.configure(inc_mode='lma', block_size=bs)
            coords, elem = meshes.square_p1(40)
            fvals = np.sin(np.pi * coords[:, 0]) * np.sin(np.pi * coords[:, 1])
            gm, gb, _ = _p1(op2, coords, elem, fvals)
            mats.append((gm.array.copy(), gb.data_ro.copy()))
        om, ob, _ = _p1(seq, coords, elem, fvals)
        np.testing.assert_array_equal(mats[0][0], om.array)
        np.testing.assert_array_equal(mats[0][0], mats[1][0])
        np.testing.assert_array_equal(mats[0][1], mats[1][1])
        assert rel_err(mats[0][1], ob.data) < 1e-15
        _clear_consts(op2)
        grid = meshes.airfoil_grid(30, 16, 5)
        G = airfoil.build(op2, 30, 16, 5, grid=grid)
        O = airfoil.build(seq, 30, 16, 5, grid=grid)
        for api, A in ((op2, G), (seq, O)):
            airfoil.save_soln(api, A)
            airfoil.adt_calc(api, A)
            airfoil.res_calc(api, A)
            airfoil.bres_calc(api, A)
        np.testing.assert_array_equal(G.p_res.data_ro, O.p_res.data)
    finally:
        cfg.configure(inc_mode=old[0], block_size=old[1])
        _clear_consts(op2)


def test_two_phase_kahan_precision_form(op2):
    """FP32 element kernels with FP64 Kahan accumulation (inc_mode='lma',
    kahan=True): the P2 stiffness and mass Mats within the FP32 element
    error of the FP64 oracle, and equal to the uncompensated sum within
    rounding."""
    from pyop2_b200 import configuration as cfg
    from pyop2_b200.workloads import fem
    old = (cfg.cfg['inc_mode'], cfg.cfg['kahan'])
    try:
        out = {}
        for kahan in (True, False):
            cfg.configure(inc_mode='lma', kahan=kahan)
            P = fem.build_p2(op2, 12, seed=3, precision="f32")
            fem.assemble_p2(op2, P)
            out[kahan] = (P.K.array.copy(), P.M.array.copy())
        Q = fem.build_p2(seq, 12, seed=3, precision="f64")
        fem.assemble_p2(seq, Q)
        assert rel_err(out[True][0], Q.K.array) < 1e-5
        assert rel_err(out[True][1], Q.M.array) < 1e-5
        assert rel_err(out[True][0], out[False][0]) < 1e-14
    finally:
        cfg.configure(inc_mode=old[0], kahan=old[1])


@pytest.mark.parametrize("opts", [dict(programmatic_launch=True), dict(fmad_inc=True),
                                  dict(staged_tl_regs=True), dict(read_replicas=True,
                                                                  replica_min_size=0),
                                  dict(staged_pair=2), dict(staged_pair=2, partition_size=512),
                                  dict(read_replicas=True, replica_min_size=0,
                                       gathered_replicas=True),
                                  dict(staged_bank_slots=True),
                                  dict(staged_bank_slots=True, staged_tl_regs=True)])
def test_airfoil_chain_launch_options_match_oracle(op2, opts):
    """The launch-level options on the staged airfoil chain: programmatic
    dependent launch (every stub waits for its predecessor), multiply-add
    contraction in INC-form loops, target ids in registers, READ replicas on
    small sets, two elements per thread in the staged passes (odd and even
    pass counts), element-gathered READ copies, bank-aware slot numbering
    (padding slots skipped by the copy and the flush); q and rms within
    1e-12 of the oracle after three iterations."""
    from pyop2_b200 import b200
    from pyop2_b200 import configuration as cfg
    from pyop2_b200._lib import call
    _clear_consts(op2)
    cfg.configure(staged_min_size=0, **opts)
    if opts.get("programmatic_launch"):
        call("op2b_set_programmatic_launch", 1)
    try:
        grid = meshes.airfoil_grid(60, 30, 4)
        G = airfoil.build(op2, 60, 30, 4, grid=grid)
        O = airfoil.build(seq, 60, 30, 4, grid=grid)
        for _ in range(3):
            gr = airfoil.iteration(op2, G)
            orr = airfoil.iteration(seq, O)
        assert rel_err(G.p_q.data_ro, O.p_q.data) < TOL
        assert rel_err(gr.data, orr.data) < TOL
        if opts.get("read_replicas"):
            assert any(bl.replicas for bl in b200.ParLoop._bound_cache.values()
                       if bl.spec.kernel_name == "adt_calc")
        if opts.get("gathered_replicas"):
            assert any(bl.spec.gathered for bl in b200.ParLoop._bound_cache.values()
                       if bl.spec.kernel_name == "adt_calc")
    finally:
        call("op2b_set_programmatic_launch", 0)
        _clear_consts(op2)


@pytest.mark.parametrize("split", ["3x2", "2x2", "6x1"])
def test_p2_itspace_split_matches_oracle(op2, split):
    """Mat assembly with the 6x6 local positions split across warps: both
    Mats of the fused P2 loop within 1e-12 of the oracle."""
    from pyop2_b200 import configuration as cfg
    from pyop2_b200.workloads import fem
    cfg.configure(itspace_split=split)
    G, O = fem.build_p2(op2, 12, seed=3), fem.build_p2(seq, 12, seed=3)
    fem.assemble_p2(op2, G)
    fem.assemble_p2(seq, O)
    assert rel_err(G.K.array, O.K.array) < TOL
    assert rel_err(G.M.array, O.M.array) < TOL


def test_gather_form_is_bit_exact(op2):
    """The gather form adds each target's contributions in the sequential
    backend's order (element order, then map index) with the same
    arithmetic, so res_calc and bres_calc equal the oracle bit for bit."""
    from pyop2_b200 import b200
    from pyop2_b200 import configuration as cfg
    _clear_consts(op2)
    cfg.configure(inc_mode="gather", staged_min_size=0)
    try:
        grid = meshes.airfoil_grid(60, 30, 6)
        G = airfoil.build(op2, 60, 30, 6, grid=grid)
        O = airfoil.build(seq, 60, 30, 6, grid=grid)
        for api, A in ((op2, G), (seq, O)):
            airfoil.save_soln(api, A)
            airfoil.adt_calc(api, A)
            airfoil.res_calc(api, A)
            airfoil.bres_calc(api, A)
        assert {bl.spec.mode for bl in b200.ParLoop._bound_cache.values()
                if bl.iterset is G.edges or bl.iterset is G.bedges} == {"gather"}
        np.testing.assert_array_equal(G.p_res.data_ro, O.p_res.data)
    finally:
        _clear_consts(op2)


@pytest.mark.parametrize("split", ["", "3x2"])
def test_compact_slot_tables_match_oracle(op2, split):
    """Mat assembly through the compact in-row slot tables (one 64-bit word
    of in-row positions per element and local row), alone and with the
    local positions split across warps: P2 stiffness and mass within 1e-12
    of the oracle, and a batch of P1 meshes against the oracle too."""
    from pyop2_b200 import b200, batch
    from pyop2_b200 import configuration as cfg
    from pyop2_b200.workloads import batching, fem
    cfg.configure(mat_slots_rel=True, itspace_split=split)
    G, O = fem.build_p2(op2, 12, seed=5), fem.build_p2(seq, 12, seed=5)
    fem.assemble_p2(op2, G)
    fem.assemble_p2(seq, O)
    assert any(bl.spec.mat_slots_rel for bl in b200.ParLoop._bound_cache.values()
               if bl.spec.kernel_name == G.k_km.name)
    assert rel_err(G.K.array, O.K.array) < TOL
    assert rel_err(G.M.array, O.M.array) < TOL
    probs = batching.build(op2, batching.mesh_shapes(6, seed=9), seed=9)
    mass, stiff, _ = batching.instances(op2, probs)
    for insts in (mass, stiff):
        batch.BatchLoop(insts, block_size=128).launch()
    for P in probs:
        Q = fem.build_p1(seq, 0, coords=P.coords.data_ro, elem=P.elem_node.values, stiffness=True)
        fem.assemble_p1(seq, Q)
        fem.assemble_p1_stiffness(seq, Q)
        assert rel_err(P.mat.array, Q.mat.array) < TOL
        assert rel_err(P.stiff.array, Q.stiff.array) < TOL
