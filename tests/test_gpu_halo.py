"""Partitioned execution on the device (b200 par_loop over Sets with four
sizes and Halos; pyop2/sequential.py:96-117, pyop2/base.py:797-835): the
halo pack / unpack kernels against numpy, element-range launches with the
reference's Global semantics, and the airfoil problem split over two and
three ranks held by one process (LocalComm, ranks stepped together; their
kernels never wait on one another) against the sequential oracle on the
undivided mesh."""

import os
import sys

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
TOL = 1e-12


@pytest.fixture
def op2(backend):
    from pyop2_b200 import op2 as _op2
    return _op2


def _clear_consts():
    from pyop2_b200 import base
    for c in list(base.Const._defs):
        c.remove_from_namespace()


@pytest.mark.parametrize("dtype,dim,soa", [(np.float64, 4, False), (np.float64, 3, True),
                                           (np.int8, 3, False), (np.int32, 1, False)])
def test_halo_pack_unpack_match_numpy(op2, dtype, dim, soa):
    from pyop2_b200 import b200
    n = 1000
    rng = np.random.default_rng(5)
    s = op2.Set(n, dim, "s")
    vals = rng.integers(0, 100, size=(n, dim)).astype(dtype)
    d = op2.Dat(s, vals.copy(), dtype, "d", soa=soa)
    rows = b200._DatRows(d)
    idx = rng.choice(n, 300, replace=False).astype(np.int32)
    buf = rows.pack(idx)
    got = buf.to_host().reshape(dim, 300).T if soa else buf.to_host().reshape(300, dim)
    np.testing.assert_array_equal(got, vals[idx])
    dst = rng.choice(n, 300, replace=False).astype(np.int32)
    rows.unpack(dst, buf)
    want = vals.copy()
    want[dst] = vals[idx]
    np.testing.assert_array_equal(d.data_ro.reshape(n, dim), want)


def test_partitioned_set_runs_core_owned_and_exec_ranges(op2):
    """One rank, sizes (core, owned, exec, total) = (3, 6, 8, 10): an
    indirect loop that increments through a Map runs the execute halo too,
    while its Global reduction keeps the owned elements' sum only
    (pyop2/base.py:216-249); a direct loop runs the owned elements."""
    s = op2.Set([3, 6, 8, 10], 1, "parts")
    t = op2.Set(10, 1, "targets")
    m = op2.Map(s, t, 1, np.arange(10, dtype=np.int32), "ident")
    out = op2.Dat(t, np.zeros(10), np.float64, "out")
    g = op2.Global(1, 0.0, np.float64, "g")
    k = op2.Kernel("void k(double *o, double *g, double *v) { o[0] += v[0]; g[0] += v[0]; }", "k")
    v = op2.Dat(s, np.arange(1.0, 11.0), np.float64, "v")
    op2.par_loop(k, s, out(m[0], op2.INC), g(op2.INC), v(op2.IdentityMap, op2.READ))
    np.testing.assert_array_equal(out.data_ro.ravel(), [1, 2, 3, 4, 5, 6, 7, 8, 0, 0])
    assert g.data[0] == 21.0
    kd = op2.Kernel("void kd(double *v, double *g) { v[0] *= 2.0; g[0] += 1.0; }", "kd")
    h = op2.Global(1, 0.0, np.float64, "h")
    op2.par_loop(kd, s, v(op2.IdentityMap, op2.RW), h(op2.INC))
    np.testing.assert_array_equal(v.data_ro.ravel(), [2, 4, 6, 8, 10, 12, 7, 8, 9, 10])
    assert h.data[0] == 6.0


class _Recorder(object):
    """The op2 API with par_loop recorded instead of run."""

    def __init__(self, op2):
        self._op2, self.calls = op2, []

    def __getattr__(self, name):
        return getattr(self._op2, name)

    def par_loop(self, kernel, iterset, *args):
        self.calls.append((kernel, iterset, args))


@pytest.mark.parametrize("nranks,staged_core", [(2, False), (3, False), (2, True)])
def test_partitioned_airfoil_matches_oracle(op2, nranks, staged_core):
    """staged_core: the core ranges of the INC loops in the staged form (a
    locality partition of each rank's core), the rest atomic."""
    from pyop2_b200 import b200, halo
    from pyop2_b200 import configuration as cfg
    from pyop2_b200.workloads import airfoil, meshes
    if staged_core:
        cfg.configure(staged_min_size=0)
    sys.path.insert(0, ROOT)
    from oracle import seq
    g = meshes.airfoil_grid(60, 30, 3)
    q0 = airfoil.initial_q(g.ncells, 3).reshape(-1, 4)
    for c in list(seq._CONSTS.values()):
        c.remove_from_namespace()
    O = airfoil.build(seq, 0, 0, grid=g, q0=q0.copy())
    ref_rms = [float(airfoil.iteration(seq, O).data[0]) for _ in range(3)]
    _clear_consts()
    parts = airfoil.partition_grid(g, nranks)
    comms = halo.LocalGroup(nranks).comms()
    ranks = [airfoil.build_partitioned(op2, g, parts[r], comms[r], 3, q0, consts=(r == 0))
             for r in range(nranks)]
    for A in ranks:
        assert A.edges.core_size < A.edges.size < A.edges.exec_size
    rms = []
    try:
        for _ in range(3):
            recs = [_Recorder(op2) for _ in ranks]
            outs = [airfoil.iteration(rec, A) for rec, A in zip(recs, ranks)]
            for k in range(len(recs[0].calls)):
                halo.run_lockstep([b200.par_loop_phases(kern, it, *args)
                                   for kern, it, args in (recs[r].calls[k] for r in range(nranks))])
            vals = [float(x.data[0]) for x in outs]
            assert max(vals) == min(vals)
            rms.append(vals[0])
        q = np.full((g.ncells, 4), np.nan)
        for p, A in zip(parts, ranks):
            ls = p.sets["cells"]
            q[ls.l2g[:ls.sizes[1]]] = A.p_q.data_ro[:ls.sizes[1]]
        assert rel_err(q, O.p_q.data) < TOL
        for a, b in zip(rms, ref_rms):
            assert abs(a - b) <= TOL * abs(b)
        # the partitioned loops ran in the atomic form, in element ranges,
        # with the core in the staged form where asked
        part = [bl for bl in b200.ParLoop._bound_cache.values() if bl.partitioned]
        assert all(bl.spec.mode in ("direct", "atomic") for bl in part)
        cores = [bl.core_loop for bl in part if bl.core_loop is not None]
        if staged_core:
            assert any(c.spec.kernel_name == "res_calc" and c.spec.mode == "staged" for c in cores)
        else:
            assert not cores
    finally:
        _clear_consts()


def test_torch_comm_allreduce_on_device_values(op2):
    """The NCCL communicator on one rank: the Global's device value is
    reduced through a torch tensor over the library's own memory, with the
    library's stream as torch's current stream (a one-rank group: the sum is
    the value itself, and what the execute halo adds is dropped)."""
    import socket
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    from pyop2_b200 import b200, halo
    sock = socket.socket()
    sock.bind(("127.0.0.1", 0))
    port = sock.getsockname()[1]
    sock.close()
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0,
                            world_size=1, timeout=timedelta(seconds=60))
    try:
        comm = b200.torch_comm()
        assert comm.size == 1
        s = op2.Set([3, 6, 8, 8], 1, "tc_parts", halo=op2.Halo([[]], [[]], comm=comm))
        t = op2.Set(8, 1, "tc_targets")
        m = op2.Map(s, t, 1, np.arange(8, dtype=np.int32), "tc_ident")
        out = op2.Dat(t, np.zeros(8), np.float64, "tc_out")
        v = op2.Dat(s, np.arange(1.0, 9.0), np.float64, "tc_v")
        g = op2.Global(1, 0.5, np.float64, "tc_g")
        k = op2.Kernel("void k(double *o, double *g, double *v) { o[0] += v[0]; g[0] += v[0]; }",
                       "k")
        op2.par_loop(k, s, out(m[0], op2.INC), g(op2.INC), v(op2.IdentityMap, op2.READ))
        assert g.data[0] == 21.5
        np.testing.assert_array_equal(out.data_ro.ravel(), np.arange(1.0, 9.0))
        # a device buffer seen as a torch tensor is the same memory
        buf = b200._DeviceHaloBuffer.alloc(32, np.float64, (4,))
        buf.from_host(np.arange(4.0))
        t4 = buf.tensor()
        b200.synchronize()
        assert t4.device.type == "cuda" and t4.cpu().tolist() == [0.0, 1.0, 2.0, 3.0]
        req = halo.GlobalReduction(buf, comm, "max").begin()
        req.wait()
        b200.synchronize()
        np.testing.assert_array_equal(buf.to_host(), np.arange(4.0))
    finally:
        dist.destroy_process_group()


def test_partitioned_p1_rhs_matches_oracle(op2):
    """P1 RHS assembly (iteration-space INC through a Map, vector-map READ)
    over a mesh split across two ranks on one GPU, then a reduction over the
    owned nodes: owned rows of b and the all-reduced sum equal the oracle's
    on the undivided mesh."""
    from pyop2_b200 import b200, halo, partition
    from pyop2_b200.workloads import fem
    sys.path.insert(0, ROOT)
    from oracle import seq
    coords, elem = fem.square_p1(24)
    O = fem.build_p1(seq, 24)
    seq.par_loop(O.k_rhs, O.elements(3), O.b(O.elem_node[seq.i[0]], seq.INC),
                 O.coords(O.elem_vnode, seq.READ), O.f(O.elem_node, seq.READ))
    ne, nn = len(elem), len(coords)
    cx = coords[elem, 0].mean(axis=1)
    own_e = (cx > np.median(cx)).astype(np.int64)
    first = np.full(nn, ne, np.int64)
    np.minimum.at(first, elem.ravel(), np.repeat(np.arange(ne), 3))
    parts = partition.partition({"nodes": nn, "elements": ne},
                                {"elem_node": ("elements", "nodes", elem)},
                                {"elements": own_e, "nodes": own_e[first]}, 2)
    comms = halo.LocalGroup(2).comms()
    f_all = np.sin(np.pi * coords[:, 0]) * np.sin(np.pi * coords[:, 1])
    k_sum = op2.Kernel("void s(double *b, double *t) { t[0] += b[0]; }", "s")
    ranks = []
    for r, p in enumerate(parts):
        S = p.sets

        def mkset(name, dim):
            ls = S[name]
            return op2.Set(list(ls.sizes), dim, name, halo=op2.Halo(ls.sends, ls.receives, comm=comms[r]))
        nodes, vnodes, elements = mkset("nodes", 1), mkset("nodes", 2), mkset("elements", 1)
        lv = p.maps["elem_node"][2]
        en = op2.Map(elements, nodes, 3, lv, "en")
        evn = op2.Map(elements, vnodes, 3, lv, "evn")
        c = op2.Dat(vnodes, S["nodes"].local_rows(coords), np.float64, "c")
        f = op2.Dat(nodes, S["nodes"].local_rows(f_all), np.float64, "f")
        b = op2.Dat(nodes, np.zeros(S["nodes"].sizes[3]), np.float64, "b")
        for d in (c, f, b):
            d.needs_halo_update = False
        ranks.append((nodes, elements, en, evn, c, f, b, op2.Global(1, 0.0, np.float64, "t")))
    k_rhs = op2.Kernel(fem.P1_RHS, "p1_rhs")
    halo.run_lockstep([b200.par_loop_phases(k_rhs, el(3), b(en[op2.i[0]], op2.INC),
                                            c(evn, op2.READ), f(en, op2.READ))
                       for nodes, el, en, evn, c, f, b, t in ranks])
    halo.run_lockstep([b200.par_loop_phases(k_sum, nodes, b(op2.IdentityMap, op2.READ), t(op2.INC))
                       for nodes, el, en, evn, c, f, b, t in ranks])
    got = np.full(nn, np.nan)
    for p, (nodes, el, en, evn, c, f, b, t) in zip(parts, ranks):
        ls = p.sets["nodes"]
        got[ls.l2g[:ls.sizes[1]]] = b.data_ro.ravel()[:ls.sizes[1]]
        assert abs(t.data[0] - O.b.data.sum()) <= TOL * abs(O.b.data).sum()
    assert rel_err(got, O.b.data) < TOL


@pytest.mark.parametrize("mode,want", [("MIN", 1.0), ("MAX", 8.0), ("INC", 36.0)])
def test_partitioned_global_reductions_across_ranks(op2, mode, want):
    """Global MIN / MAX / INC over the owned elements of a set split across
    two ranks on one GPU: every rank holds the reduction over both ranks'
    owned elements (pyop2/base.py:216-249), and the execute halo's values
    (here the largest and smallest of all) never reach it."""
    from pyop2_b200 import b200, halo
    comms = halo.LocalGroup(2).comms()
    # rank 0 owns values 1..4, rank 1 owns 5..8; each holds an execute-halo
    # copy of one peer element with a value outside [1, 8]
    k = op2.Kernel("void r(double *o, double *g, double *v) { o[0] += 0.0; %s }" % {
        "MIN": "if (v[0] < g[0]) g[0] = v[0];", "MAX": "if (v[0] > g[0]) g[0] = v[0];",
        "INC": "g[0] += v[0];"}[mode], "r")
    ranks = []
    for r in range(2):
        own = np.arange(1.0, 5.0) + 4 * r
        vals = np.concatenate([own, [100.0 if mode != "MIN" else -100.0]])
        sends = [np.zeros(0, np.int32), np.array([3], np.int32)] if r == 0 else \
            [np.array([0], np.int32), np.zeros(0, np.int32)]
        recvs = [np.zeros(0, np.int32), np.array([4], np.int32)] if r == 0 else \
            [np.array([4], np.int32), np.zeros(0, np.int32)]
        s = op2.Set([2, 4, 5, 5], 1, "gr%d" % r, halo=op2.Halo(sends, recvs, comm=comms[r]))
        t = op2.Set(5, 1, "gt%d" % r)
        m = op2.Map(s, t, 1, np.arange(5, dtype=np.int32), "gm%d" % r)
        out = op2.Dat(t, np.zeros(5), np.float64, "go%d" % r)
        v = op2.Dat(s, vals, np.float64, "gv%d" % r)
        v.needs_halo_update = False
        init = {"MIN": 1e30, "MAX": -1e30, "INC": 0.0}[mode]
        ranks.append((s, m, out, v, op2.Global(1, init, np.float64, "g%d" % r)))
    acc = {"MIN": op2.MIN, "MAX": op2.MAX, "INC": op2.INC}[mode]
    halo.run_lockstep([b200.par_loop_phases(k, s, out(m[0], op2.INC), g(acc), v(op2.IdentityMap, op2.READ))
                       for s, m, out, v, g in ranks])
    for s, m, out, v, g in ranks:
        assert g.data[0] == want
