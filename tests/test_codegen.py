"""Stub generation: every loop form of the reference's unit tests and of the
workloads generates CUDA that NVRTC compiles for sm_100a.  NVRTC needs no GPU,
so this runs on the CPU and catches generator errors before a GPU run."""

import ctypes as C
import re

import numpy as np
import pytest

from pyop2_b200 import backends, codegen


@pytest.fixture(scope="module")
def host_op2():
    """The op2 API with the B200 backend selected but no device initialised
    (the data classes are host-only until a loop runs)."""
    from pyop2_b200 import _lib, op2
    if backends.get_backend() == "pyop2_b200.void":
        backends.set_backend("b200")
    _lib.load()
    return op2


def nvrtc_compile(spec, extra=(), want_log=False):
    from pyop2_b200 import _lib
    src, layout, _ = codegen.generate(spec)
    opts = codegen.nvrtc_options(extra=extra)
    arr = (C.c_char_p * len(opts))(*[o.encode() for o in opts])
    out, n = C.c_void_p(), C.c_uint64()
    log = C.create_string_buffer(1 << 16)
    rc = _lib._lib.op2b_nvrtc_compile(src.encode(), b"stub.cu", arr, len(opts), C.byref(out),
                                      C.byref(n), log, len(log))
    assert rc == 0, _lib.last_error() + "\n" + src
    _lib._lib.op2b_cubin_free(out)
    if want_log:
        return src, layout, n.value, log.value.decode()
    return src, layout, n.value


def spec_of(op2, kernel, itspace, *args):
    from pyop2_b200 import b200
    return b200.loop_spec(b200.ParLoop(kernel, itspace, *args))["spec"]


def test_direct_forms(host_op2):
    op2 = host_op2
    s1, s2 = op2.Set(10, 1), op2.Set(10, 2)
    x = op2.Dat(s1, np.zeros(10, np.uint32), np.uint32)
    y = op2.Dat(s2, np.zeros(20, np.uint32), np.uint32)
    soa = op2.Dat(s2, np.zeros(20, np.uint32), np.uint32, soa=True)
    g = op2.Global(1, 0, np.uint32)
    g2 = op2.Global(2, (0, 0), np.float64)
    for acc in (op2.READ, op2.WRITE, op2.RW, op2.INC):
        nvrtc_compile(spec_of(op2, op2.Kernel("void k(unsigned int *a) { }", "k"), s1, x(op2.IdentityMap, acc)))
    for acc in (op2.INC, op2.MIN, op2.MAX, op2.READ):
        src, _, _ = nvrtc_compile(spec_of(op2, op2.Kernel("void k(unsigned int *a, unsigned int *g) { }", "k"),
                                          s1, x(op2.IdentityMap, op2.READ), g(acc)))
    nvrtc_compile(spec_of(op2, op2.Kernel("void k(unsigned int *a, double *g) { }", "k"), s2,
                          y(op2.IdentityMap, op2.RW), g2(op2.INC)))
    src, _, _ = nvrtc_compile(spec_of(op2, op2.Kernel(
        "void k(unsigned int *a) { OP2_STRIDE(a, 0) = 1; OP2_STRIDE(a, 1) = 2; }", "k"), s2,
        soa(op2.IdentityMap, op2.WRITE)))
    assert "op2b_store_soa" in src


def test_indirect_forms(host_op2, golden_matrices):
    op2 = host_op2
    el, nd, vnd = op2.Set(2), op2.Set(4), op2.Set(4, 2)
    emap = np.asarray(golden_matrices["elem_node_map"], np.int32)
    en = op2.Map(el, nd, 3, emap, "en")
    evn = op2.Map(el, vnd, 3, emap, "evn")
    coords = op2.Dat(vnd, np.zeros(8))
    f = op2.Dat(nd, np.zeros(4))
    b = op2.Dat(nd, np.zeros(4))
    bv = op2.Dat(vnd, np.zeros(8))
    mat = op2.Mat(op2.Sparsity((en, en)), np.float64)
    vmat = op2.Mat(op2.Sparsity((evn, evn)), np.float64)
    gl = op2.Global(1, 1.0, np.float64)
    K = {k: op2.Kernel(v["code"], v["name"]) for k, v in golden_matrices["kernels"].items()}
    srcs = []
    srcs.append(nvrtc_compile(spec_of(op2, K["mass"], el(3, 3), mat((en[op2.i[0]], en[op2.i[1]]), op2.INC),
                                      coords(evn, op2.READ)))[0])
    srcs.append(nvrtc_compile(spec_of(op2, K["mass_vector_ffc"], el(3, 3),
                                      vmat((evn[op2.i[0]], evn[op2.i[1]]), op2.INC), coords(evn, op2.READ)))[0])
    srcs.append(nvrtc_compile(spec_of(op2, K["kernel_set_vec"], el(3, 3),
                                      vmat((evn[op2.i[0]], evn[op2.i[1]]), op2.WRITE), gl(op2.READ)))[0])
    srcs.append(nvrtc_compile(spec_of(op2, K["rhs"], el, b(en, op2.INC), coords(evn, op2.READ),
                                      f(en, op2.READ)))[0])
    srcs.append(nvrtc_compile(spec_of(op2, K["rhs_ffc_itspace"], el(3), b(en[op2.i[0]], op2.INC),
                                      coords(evn, op2.READ), f(en, op2.READ)))[0])
    srcs.append(nvrtc_compile(spec_of(op2, K["rhs_ffc_vector_itspace"], el(3), bv(evn[op2.i[0]], op2.INC),
                                      coords(evn, op2.READ), bv(evn, op2.READ)))[0])
    for acc in (op2.WRITE, op2.RW, op2.READ):
        srcs.append(nvrtc_compile(spec_of(op2, op2.Kernel("void k(double *a[1], double *g) { }", "k"), el,
                                          b(en, acc), gl(op2.INC)))[0])
    assert all('extern "C" __global__' in s for s in srcs)
    assert "op2b_mass(" in srcs[0] and "op2b_rhs_ffc_itspace(" in srcs[4]
    assert "op2b_csr_find" in srcs[0]


def test_airfoil_stubs(host_op2):
    from pyop2_b200 import base
    from pyop2_b200.workloads import airfoil
    op2 = host_op2
    for c in list(base.Const._defs):
        c.remove_from_namespace()
    A = airfoil.build(op2, 6, 3, 0)
    from pyop2_b200 import b200
    loops = [
        (A.k_save, A.cells, [A.p_q(op2.IdentityMap, op2.READ), A.p_qold(op2.IdentityMap, op2.WRITE)]),
        (A.k_adt, A.cells, [A.p_x(A.pcell[k], op2.READ) for k in range(4)] +
         [A.p_q(op2.IdentityMap, op2.READ), A.p_adt(op2.IdentityMap, op2.WRITE)]),
        (A.k_res, A.edges, [A.p_x(A.pedge[0], op2.READ), A.p_x(A.pedge[1], op2.READ),
                            A.p_q(A.pevcell[0], op2.READ), A.p_q(A.pevcell[1], op2.READ),
                            A.p_adt(A.pecell[0], op2.READ), A.p_adt(A.pecell[1], op2.READ),
                            A.p_res(A.pevcell[0], op2.INC), A.p_res(A.pevcell[1], op2.INC)]),
        (A.k_bres, A.bedges, [A.p_x(A.pbedge[0], op2.READ), A.p_x(A.pbedge[1], op2.READ),
                              A.p_q(A.pbevcell[0], op2.READ), A.p_adt(A.pbecell[0], op2.READ),
                              A.p_res(A.pbevcell[0], op2.INC), A.p_bound(op2.IdentityMap, op2.READ)]),
        (A.k_update, A.cells, [A.p_qold(op2.IdentityMap, op2.READ), A.p_q(op2.IdentityMap, op2.WRITE),
                               A.p_res(op2.IdentityMap, op2.RW), A.p_adt(op2.IdentityMap, op2.READ),
                               op2.Global(1, 0.0, np.float64)(op2.INC)])]
    for k, s, args in loops:
        info = b200.loop_spec(b200.ParLoop(k, s, *args))
        src, layout, n = nvrtc_compile(info["spec"])
        assert n > 0
    for c in A.consts:
        c.remove_from_namespace()


def test_airfoil_stub_resources(host_op2):
    """ptxas's resource report for the airfoil stubs as the bench runs them
    (res_calc in the staged form): no stack frame and no spills in any, and
    the staged res_calc within 64 registers, so 8 CTAs of 128 threads stay
    resident per SM."""
    import re
    from pyop2_b200 import b200, base
    from pyop2_b200 import configuration as cfg
    from pyop2_b200.workloads import airfoil
    op2 = host_op2
    for c in list(base.Const._defs):
        c.remove_from_namespace()
    A = airfoil.build(op2, 6, 3, 0)
    cfg.configure(staged_min_size=0)
    try:
        loops = {
            "adt_calc": (A.k_adt, A.cells, [A.p_x(A.pcell[k], op2.READ) for k in range(4)] +
                         [A.p_q(op2.IdentityMap, op2.READ), A.p_adt(op2.IdentityMap, op2.WRITE)]),
            "res_calc": (A.k_res, A.edges, [A.p_x(A.pedge[0], op2.READ), A.p_x(A.pedge[1], op2.READ),
                                            A.p_q(A.pevcell[0], op2.READ), A.p_q(A.pevcell[1], op2.READ),
                                            A.p_adt(A.pecell[0], op2.READ), A.p_adt(A.pecell[1], op2.READ),
                                            A.p_res(A.pevcell[0], op2.INC), A.p_res(A.pevcell[1], op2.INC)]),
            "update": (A.k_update, A.cells, [A.p_qold(op2.IdentityMap, op2.READ),
                                             A.p_q(op2.IdentityMap, op2.WRITE),
                                             A.p_res(op2.IdentityMap, op2.RW),
                                             A.p_adt(op2.IdentityMap, op2.READ),
                                             op2.Global(1, 0.0, np.float64)(op2.INC)])}
        for name, (k, s, args) in loops.items():
            spec = b200.loop_spec(b200.ParLoop(k, s, *args))["spec"]
            if name == "res_calc":
                assert spec.mode == "staged"
            _, _, _, log = nvrtc_compile(spec, extra=["-Xptxas=-v"], want_log=True)
            m = re.search(r"(\d+) bytes stack frame, (\d+) bytes spill stores, (\d+) bytes spill loads", log)
            assert m and m.groups() == ("0", "0", "0"), (name, log)
            regs = int(re.search(r"Used (\d+) registers", log).group(1))
            if name == "res_calc":
                assert regs <= 64, (name, regs)
    finally:
        # the configuration is put back by conftest's autouse fixture
        for c in A.consts:
            c.remove_from_namespace()


def test_atomic_mode_stubs(host_op2, golden_matrices):
    """The atomic INC form of the indirect loops compiles (Dat INC through
    maps, vec maps and iteration spaces; Mat INC)."""
    op2 = host_op2
    from pyop2_b200 import b200
    from pyop2_b200 import configuration as cfg
    el, nd, vnd = op2.Set(2), op2.Set(4), op2.Set(4, 2)
    emap = np.asarray(golden_matrices["elem_node_map"], np.int32)
    en = op2.Map(el, nd, 3, emap, "en_a")
    evn = op2.Map(el, vnd, 3, emap, "evn_a")
    coords, f = op2.Dat(vnd, np.zeros(8)), op2.Dat(nd, np.zeros(4))
    b, bv = op2.Dat(nd, np.zeros(4)), op2.Dat(vnd, np.zeros(8))
    mat = op2.Mat(op2.Sparsity((en, en)), np.float64)
    vmat = op2.Mat(op2.Sparsity((evn, evn)), np.float64)
    K = {k: op2.Kernel(v["code"], v["name"]) for k, v in golden_matrices["kernels"].items()}
    cfg.configure(inc_mode="atomic", owner_mode="never")
    try:
        cases = [(K["mass"], el(3, 3), mat((en[op2.i[0]], en[op2.i[1]]), op2.INC), coords(evn, op2.READ)),
                 (K["mass_vector_ffc"], el(3, 3), vmat((evn[op2.i[0]], evn[op2.i[1]]), op2.INC),
                  coords(evn, op2.READ)),
                 (K["rhs"], el, b(en, op2.INC), coords(evn, op2.READ), f(en, op2.READ)),
                 (K["rhs_ffc_itspace"], el(3), b(en[op2.i[0]], op2.INC), coords(evn, op2.READ),
                  f(en, op2.READ)),
                 (K["rhs_ffc_vector_itspace"], el(3), bv(evn[op2.i[0]], op2.INC), coords(evn, op2.READ),
                  bv(evn, op2.READ))]
        for k, it, *args in cases:
            info = b200.loop_spec(b200.ParLoop(k, it, *args))
            assert info["spec"].mode == "atomic"
            src, layout, _ = nvrtc_compile(info["spec"])
            assert "op2b_atomic" in src and "blkmap" not in layout.fields
        # a Mat WRITE still needs the coloured form
        info = b200.loop_spec(b200.ParLoop(K["kernel_set"], el(3, 3), mat((en[op2.i[0]], en[op2.i[1]]), op2.WRITE),
                                           op2.Global(1, 1.0, np.float64)(op2.READ)))
        assert info["spec"].mode == "plan"
    finally:
        cfg.configure(inc_mode="staged", owner_mode="never")


def test_staged_mode_stubs(host_op2, golden_matrices):
    """The staged form (locality partition, shared-memory INC accumulation)
    compiles for Dat INC through indexed, vec-map and iteration-space args;
    Maps with equal values share one staged target list; loops without an
    indirect INC or with Mats run in the atomic form instead."""
    op2 = host_op2
    from pyop2_b200 import b200, base
    from pyop2_b200 import configuration as cfg
    from pyop2_b200.workloads import airfoil
    el, nd, vnd = op2.Set(2), op2.Set(4), op2.Set(4, 2)
    emap = np.asarray(golden_matrices["elem_node_map"], np.int32)
    en = op2.Map(el, nd, 3, emap, "en_s")
    evn = op2.Map(el, vnd, 3, emap, "evn_s")
    coords, f = op2.Dat(vnd, np.zeros(8)), op2.Dat(nd, np.zeros(4))
    b, bv = op2.Dat(nd, np.zeros(4)), op2.Dat(vnd, np.zeros(8))
    mat = op2.Mat(op2.Sparsity((en, en)), np.float64)
    K = {k: op2.Kernel(v["code"], v["name"]) for k, v in golden_matrices["kernels"].items()}
    for c in list(base.Const._defs):
        c.remove_from_namespace()
    A = airfoil.build(op2, 6, 3, 0)
    cfg.configure(inc_mode="staged", owner_mode="never", staged_min_size=0)
    try:
        cases = [(K["rhs"], el, b(en, op2.INC), coords(evn, op2.READ), f(en, op2.READ)),
                 (K["rhs_ffc_itspace"], el(3), b(en[op2.i[0]], op2.INC), coords(evn, op2.READ),
                  f(en, op2.READ)),
                 (K["rhs_ffc_vector_itspace"], el(3), bv(evn[op2.i[0]], op2.INC), coords(evn, op2.READ),
                  bv(evn, op2.READ)),
                 (A.k_res, A.edges, A.p_x(A.pedge[0], op2.READ), A.p_x(A.pedge[1], op2.READ),
                  A.p_q(A.pevcell[0], op2.READ), A.p_q(A.pevcell[1], op2.READ),
                  A.p_adt(A.pecell[0], op2.READ), A.p_adt(A.pecell[1], op2.READ),
                  A.p_res(A.pevcell[0], op2.INC), A.p_res(A.pevcell[1], op2.INC)),
                 (A.k_bres, A.bedges, A.p_x(A.pbedge[0], op2.READ), A.p_x(A.pbedge[1], op2.READ),
                  A.p_q(A.pbevcell[0], op2.READ), A.p_adt(A.pbecell[0], op2.READ),
                  A.p_res(A.pbevcell[0], op2.INC), A.p_bound(op2.IdentityMap, op2.READ))]
        for k, it, *args in cases:
            spec = b200.loop_spec(b200.ParLoop(k, it, *args))["spec"]
            assert spec.mode == "staged", k.name
            src, layout, _ = nvrtc_compile(spec)
            assert "rg_thrcol" in layout.fields and "op2b_atomic_add(p.d" in src
            R = spec.region
            # en and evn (one connectivity, two target DataSets) stage one list
            assert len(R["stage_arity"]) == (2 if k is A.k_res or k is A.k_bres else 1), k.name
        res = b200.loop_spec(b200.ParLoop(*cases[3]))["spec"]
        cells = res.region["map_stage"][res.args[6].mslot]
        nodes = res.region["map_stage"][res.args[0].mslot]
        assert res.region["inc_pairs"] == [(res.args[6].slot, cells, "double", 4)]
        assert res.region["inc_stages"] == [cells]
        # x through pedge, q through pevcell, adt through pecell: staged READ rows
        assert sorted(res.region["read_pairs"]) == sorted([(res.args[0].slot, nodes, "double", 2),
                                                           (res.args[2].slot, cells, "double", 4),
                                                           (res.args[4].slot, cells, "double", 1)])
        # below staged_min_size: the atomic form
        cfg.configure(staged_min_size=1 << 30)
        assert b200.loop_spec(b200.ParLoop(*cases[3]))["spec"].mode == "atomic"
        cfg.configure(staged_min_size=0)
        # no indirect INC / a Mat: the atomic form
        adt = b200.loop_spec(b200.ParLoop(A.k_adt, A.cells, *([A.p_x(A.pcell[k], op2.READ) for k in range(4)] +
                             [A.p_q(op2.IdentityMap, op2.READ), A.p_adt(op2.IdentityMap, op2.WRITE)])))
        assert adt["spec"].mode == "atomic"
        m = b200.loop_spec(b200.ParLoop(K["mass"], el(3, 3), mat((en[op2.i[0]], en[op2.i[1]]), op2.INC),
                                        coords(evn, op2.READ)))
        assert m["spec"].mode == "atomic"
    finally:
        cfg.configure(inc_mode="staged", owner_mode="never", staged_min_size=262144)
        for c in A.consts:
            c.remove_from_namespace()


def test_owner_mode_stubs(host_op2, golden_matrices):
    """Owner-computes stubs: scalar Mat INC/WRITE, 1-d iteration-space Dat
    INC, indexed / vec-map Dat INC (owner_mode='always'), with and without
    Kahan compensation."""
    op2 = host_op2
    from pyop2_b200 import b200
    from pyop2_b200 import configuration as cfg
    el, nd, vnd = op2.Set(2), op2.Set(4), op2.Set(4, 2)
    emap = np.asarray(golden_matrices["elem_node_map"], np.int32)
    en = op2.Map(el, nd, 3, emap, "en_o")
    evn = op2.Map(el, vnd, 3, emap, "evn_o")
    coords, f = op2.Dat(vnd, np.zeros(8)), op2.Dat(nd, np.zeros(4))
    b = op2.Dat(nd, np.zeros(4))
    mat = op2.Mat(op2.Sparsity((en, en)), np.float64)
    g = op2.Global(1, 1.0, np.float64)
    K = {k: op2.Kernel(v["code"], v["name"]) for k, v in golden_matrices["kernels"].items()}
    cases = [(K["mass"], el(3, 3), mat((en[op2.i[0]], en[op2.i[1]]), op2.INC), coords(evn, op2.READ)),
             (K["kernel_set"], el(3, 3), mat((en[op2.i[0]], en[op2.i[1]]), op2.WRITE), g(op2.READ)),
             (K["rhs_ffc_itspace"], el(3), b(en[op2.i[0]], op2.INC), coords(evn, op2.READ), f(en, op2.READ)),
             (K["rhs"], el, b(en, op2.INC), coords(evn, op2.READ), f(en, op2.READ))]
    for kahan in (False, True):
        cfg.configure(owner_mode="always", kahan=kahan)
        try:
            for k, it, *args in cases:
                info = b200.loop_spec(b200.ParLoop(k, it, *args), mat_nnz_max=16)
                assert info["spec"].mode == "owner", k.name
                src, layout, _ = nvrtc_compile(info["spec"])
                assert "inc_list" in layout.fields
                assert ("comp[" in src) == kahan
        finally:
            cfg.configure(owner_mode="never", kahan=False)
    # a Global reduction forbids owner-computes
    red = op2.Global(1, 0.0, np.float64)
    info = b200.loop_spec(b200.ParLoop(op2.Kernel("void kg(double *b, double *g) { }", "kg"), el,
                                       b(en[0], op2.INC), red(op2.INC)))
    assert info["spec"].mode != "owner"


def test_param_layout_offsets():
    spec = codegen.LoopSpec("k", "void k(double *a) {}", (), [], [("double", False)], [3], [], [], [],
                            True, [], 256, False)
    L = codegen.ParamLayout(spec)
    assert L.COL_OFFSET == 8
    assert L.nbytes == 32 + 8 * len(L.fields)
    packed = L.pack(100, 0, 100, {"d0": 0x1000, "m0": 0x2000})
    assert len(packed) == L.nbytes


def _batched(spec, ept=2):
    import copy
    from pyop2_b200 import b200
    s = copy.copy(spec)
    s.batch = ept
    return s


def test_batched_forms(host_op2):
    """Batched stubs (one launch over many instances): direct loops with
    Global INC / MIN / MAX, atomic indirect INC into Dats and a Mat."""
    from pyop2_b200 import b200
    op2 = host_op2
    s1, s2 = op2.Set(10, 1), op2.Set(10, 2)
    x = op2.Dat(s1, np.zeros(10), np.float64)
    y = op2.Dat(s2, np.zeros(20), np.float64)
    g = op2.Global(1, 0.0, np.float64)
    g3 = op2.Global(3, (0.0, 0.0, 0.0), np.float64)
    k = op2.Kernel("void k(double *a, double *g) { g[0] += a[0]; }", "k")
    for acc in (op2.INC, op2.MIN, op2.MAX, op2.READ):
        spec = b200.loop_spec(b200.ParLoop(k, s1, x(op2.IdentityMap, op2.READ), g(acc)),
                              inc_mode='atomic', owner_mode='never')["spec"]
        src, _, _ = nvrtc_compile(_batched(spec))
        assert "op2b_k_batch" in src and "op2b_k_batch_fin" in src
    spec = b200.loop_spec(b200.ParLoop(op2.Kernel("void k3(double *a, double *g) { }", "k3"), s2,
                                       y(op2.IdentityMap, op2.RW), g3(op2.INC)),
                          inc_mode='atomic', owner_mode='never')["spec"]
    nvrtc_compile(_batched(spec, 4))
    # indirect: vec-map READ, itspace INC, Mat INC
    e = op2.Set(4, 1)
    n = op2.Set(6, 1)
    vn = op2.Set(6, 2)
    em = op2.Map(e, n, 3, np.array([0, 1, 2, 1, 2, 3, 2, 3, 4, 3, 4, 5], np.int32))
    evm = op2.Map(e, vn, 3, np.array([0, 1, 2, 1, 2, 3, 2, 3, 4, 3, 4, 5], np.int32))
    xy = op2.Dat(vn, np.zeros(12), np.float64)
    b = op2.Dat(n, np.zeros(6), np.float64)
    sp = op2.Sparsity((em, em))
    mat = op2.Mat(sp, np.float64)
    km = op2.Kernel("void km(double A[1][1], double *x[2], int j, int k) { A[0][0] += x[j][0] * x[k][1]; }", "km")
    spec = b200.loop_spec(b200.ParLoop(km, e(3, 3), mat((em[op2.i[0]], em[op2.i[1]]), op2.INC),
                                       xy(evm, op2.READ)), inc_mode='atomic', owner_mode='never',
                          mat_nnz_max=8)["spec"]
    assert spec.mode == "atomic"
    src, _, _ = nvrtc_compile(_batched(spec, 1))
    assert "op2b_km_batch_fin" in src
    kr = op2.Kernel("void kr(double *b, double *x[2], int j) { b[0] += x[j][0]; }", "kr")
    spec = b200.loop_spec(b200.ParLoop(kr, e(3), b(em[op2.i[0]], op2.INC), xy(evm, op2.READ)),
                          inc_mode='atomic', owner_mode='never')["spec"]
    nvrtc_compile(_batched(spec, 2))


def test_batch_layout_fields(host_op2):
    from pyop2_b200 import b200
    op2 = host_op2
    s1 = op2.Set(10, 1)
    x = op2.Dat(s1, np.zeros(10), np.float64)
    g = op2.Global(1, 0.0, np.float64)
    h = op2.Global(1, 0.0, np.float64)
    k = op2.Kernel("void k(double *a, double *g, double *h) { }", "k")
    spec = b200.loop_spec(b200.ParLoop(k, s1, x(op2.IdentityMap, op2.READ), g(op2.INC), h(op2.READ)),
                          inc_mode='atomic', owner_mode='never')["spec"]
    lay = codegen.BatchLayout(spec)
    assert lay.fields == ["segs", "tiles", "tile_first", "ntiles", "nsegs", "gpart0"]
    assert lay.nbytes == 48


def test_two_phase_forms(host_op2):
    """Two-phase (inc_mode='lma') stubs: Mat INC, vec-map and indexed Dat INC
    write contribution arrays instead of adding."""
    from pyop2_b200 import b200
    op2 = host_op2
    e = op2.Set(4, 1)
    n = op2.Set(6, 1)
    vn = op2.Set(6, 2)
    em = op2.Map(e, n, 3, np.array([0, 1, 2, 1, 2, 3, 2, 3, 4, 3, 4, 5], np.int32))
    evm = op2.Map(e, vn, 3, np.array([0, 1, 2, 1, 2, 3, 2, 3, 4, 3, 4, 5], np.int32))
    xy = op2.Dat(vn, np.zeros(12), np.float64)
    b = op2.Dat(n, np.zeros(6), np.float64)
    mat = op2.Mat(op2.Sparsity((em, em)), np.float64)
    km = op2.Kernel("void km(double A[1][1], double *x[2], int j, int k) { A[0][0] += x[j][0]; }", "km")
    spec = b200.loop_spec(b200.ParLoop(km, e(3, 3), mat((em[op2.i[0]], em[op2.i[1]]), op2.INC),
                                       xy(evm, op2.READ)), inc_mode='lma', owner_mode='never',
                          mat_nnz_max=8)["spec"]
    assert spec.mode == "lma"
    src, layout, _ = nvrtc_compile(spec)
    assert "p.lm0[" in src and "lm0" in layout.fields and "op2b_atomic" not in src.split("op2b_user")[-1]
    kv = op2.Kernel("void kv(double *b[1], double *x[2]) { b[0][0] += x[0][0]; b[2][0] += 1.0; }", "kv")
    spec = b200.loop_spec(b200.ParLoop(kv, e, b(em, op2.INC), xy(evm, op2.READ)),
                          inc_mode='lma', owner_mode='never')["spec"]
    assert spec.mode == "lma"
    src, layout, _ = nvrtc_compile(spec)
    assert "p.ld0" in src and "ld0" in layout.fields
    ki = op2.Kernel("void ki(double *b0, double *b1) { *b0 += 1.0; *b1 += 2.0; }", "ki")
    spec = b200.loop_spec(b200.ParLoop(ki, e, b(em[0], op2.INC), b(em[2], op2.INC)),
                          inc_mode='lma', owner_mode='never')["spec"]
    assert spec.mode == "lma"
    nvrtc_compile(spec)
    # the same map index twice in one loop: no two-phase form
    spec = b200.loop_spec(b200.ParLoop(ki, e, b(em[0], op2.INC), b(em[0], op2.INC)),
                          inc_mode='lma', owner_mode='never')["spec"]
    assert spec.mode == "plan"


def test_gather_form_of_the_airfoil_flux_loop(host_op2):
    """The gather form (thread per target over the owner Map's incidence):
    res_calc's two INC args through one Map qualify; a Global reduction or a
    second INC Map does not (those loops keep another form)."""
    from pyop2_b200 import configuration as cfg
    from pyop2_b200.workloads import airfoil
    op2 = host_op2
    cfg.configure(inc_mode="gather", staged_min_size=0)
    A = airfoil.build(op2, 8, 4, 0, consts=False)
    op2.Const(1, 1.4, "gam", np.float64), op2.Const(1, 0.4, "gm1", np.float64)
    op2.Const(1, 0.05, "eps", np.float64), op2.Const(1, 0.9, "cfl", np.float64)
    op2.Const(4, airfoil.freestream(), "qinf", np.float64)
    try:
        spec = spec_of(op2, A.k_res, A.edges,
                       A.p_x(A.pedge[0], op2.READ), A.p_x(A.pedge[1], op2.READ),
                       A.p_q(A.pevcell[0], op2.READ), A.p_q(A.pevcell[1], op2.READ),
                       A.p_adt(A.pecell[0], op2.READ), A.p_adt(A.pecell[1], op2.READ),
                       A.p_res(A.pevcell[0], op2.INC), A.p_res(A.pevcell[1], op2.INC))
        assert spec.mode == "gather"
        src, layout, _ = nvrtc_compile(spec)
        assert "inc_order" in layout.fields and "atomic" not in src.split("op2b_res_calc")[-1]
        for kahan in (False, True):
            cfg.configure(kahan=kahan)
            nvrtc_compile(spec_of(op2, A.k_res, A.edges,
                                  A.p_x(A.pedge[0], op2.READ), A.p_x(A.pedge[1], op2.READ),
                                  A.p_q(A.pevcell[0], op2.READ), A.p_q(A.pevcell[1], op2.READ),
                                  A.p_adt(A.pecell[0], op2.READ), A.p_adt(A.pecell[1], op2.READ),
                                  A.p_res(A.pevcell[0], op2.INC), A.p_res(A.pevcell[1], op2.INC)))
        rms = op2.Global(1, 0.0, np.float64, "rms")
        k = op2.Kernel("void k(double *a, double *b, double *g) { a[0] += 1.0; b[0] += 1.0; g[0] += 1.0; }", "k")
        spec2 = spec_of(op2, k, A.edges, A.p_adt(A.pecell[0], op2.INC), A.p_adt(A.pecell[1], op2.INC),
                        rms(op2.INC))
        assert spec2.mode != "gather"
    finally:
        from pyop2_b200 import base
        for c in list(base.Const._defs):
            c.remove_from_namespace()


def test_batched_coloured_form_compiles(host_op2):
    """The coloured batched stub (a plan per instance, one launch per block
    colour, thread colours inside a block) for the batching workload's three
    loops: P1 mass and stiffness into Mats, RHS INC into a Dat."""
    from pyop2_b200 import codegen as cg
    from pyop2_b200.workloads import fem
    op2 = host_op2
    P = fem.build_p1(op2, 4, stiffness=True)
    rows = (P.elem_node[op2.i[0]], P.elem_node[op2.i[1]])
    for k, its, args in ((P.k_mass, P.elements(3, 3), (P.mat(rows, op2.INC), P.coords(P.elem_vnode, op2.READ))),
                         (P.k_rhs, P.elements(3), (P.b(P.elem_node[op2.i[0]], op2.INC),
                                                   P.coords(P.elem_vnode, op2.READ),
                                                   P.f(P.elem_node, op2.READ)))):
        spec = spec_of(op2, k, its, *args)
        spec.mode = "plan"
        spec.batch = 1
        spec.mat_slots = any(a.kind == "mat" for a in spec.args)
        spec.mat_alias = (0,) if spec.mat_slots else ()
        src, layout, _ = nvrtc_compile(spec)
        assert "p.blkmap[td.first]" in src
        assert ("__ldg(p.ms0" in src) == spec.mat_slots
    # a fused two-Mat loop shares one slot table load per entry
    Q = fem.build_p2(op2, 2)
    rows = (Q.elem_dof[op2.i[0]], Q.elem_dof[op2.i[1]])
    spec = spec_of(op2, Q.k_km, Q.elements(6, 6), Q.K(rows, op2.INC), Q.M(rows, op2.INC),
                   Q.coords(Q.elem_vdof, op2.READ))
    assert spec.mode == "atomic" and spec.mat_alias == (0, 0) and spec.mat_per_entry
    src, _, _ = nvrtc_compile(spec)
    assert "p.ms1" not in src.split("extern \"C\"")[-1]


def test_reduction_initial_value_fields(host_op2):
    """A reduction Global of a supported type and at most four components
    gets a flag and one 8-byte word per component in the parameter block;
    the stub takes the value before the loop from them when the flag is set
    (MIN/MAX start from it, the last CTA combines the sum with it); larger
    or READ Globals keep the device value only.  Every form compiles."""
    op2 = host_op2
    s = op2.Set(10, 1)
    x = op2.Dat(s, np.zeros(10), np.float64)
    for dt, ct in ((np.float64, "double"), (np.float32, "float"), (np.int32, "int"),
                   (np.uint32, "unsigned int"), (np.int64, "long long"),
                   (np.uint64, "unsigned long long")):
        g = op2.Global(3, [0, 0, 0], dt)
        big = op2.Global(5, [0] * 5, dt)
        rd = op2.Global(1, [1], dt)
        k = op2.Kernel("void k(double *a, %s *g, %s *b, %s *r) { }" % (ct, ct, ct), "k")
        for acc in (op2.INC, op2.MIN, op2.MAX):
            src, layout, _ = nvrtc_compile(spec_of(op2, k, s, x(op2.IdentityMap, op2.READ),
                                                   g(acc), big(op2.INC), rd(op2.READ)))
            f = layout.fields
            assert ["gf0", "gv0_0", "gv0_1", "gv0_2"] == [n for n in f if n.startswith(("gf0", "gv0"))]
            assert not any(n.startswith(("gf1", "gv1", "gf2", "gv2")) for n in f)
            assert "p.gf0 != 0, i1" in src
            if acc is not op2.INC:
                assert "r1[2] = p.gf0 ?" in src
    assert not codegen.gbl_init_fields(("unsigned char", 1, "INC"))
    assert not codegen.gbl_init_fields(("double", 1, "READ"))
    assert codegen.gbl_init_fields(("double", codegen.GBL_INIT_MAX, "MAX"))
