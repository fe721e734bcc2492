"""Partitioned execution on the host (pyop2_b200/halo.py with
pyop2_b200/partition.py): the communicators, one Dat's halo exchange, one
Global's reduction, and whole airfoil runs split over ranks -- in one
process (ranks stepped together) and as two gloo processes -- against the
sequential oracle on the undivided mesh.

The loop order is the reference's (pyop2/sequential.py:96-117): exchange
start, core elements, exchange end, other owned elements, reduction start,
execute halo, reduction end.  The element ranges run on the oracle here
(the GPU path runs them as device launches in tests/test_gpu_halo.py)."""

import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

from pyop2_b200 import halo
from pyop2_b200.workloads import airfoil, meshes

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
TOL = 1e-12


# ---------------------------------------------------------------- units
def test_local_exchange_pairs_messages_in_order():
    comms = halo.LocalGroup(2).comms()
    a = [np.arange(6.0).reshape(3, 2), 10 + np.arange(6.0).reshape(3, 2)]
    rows = [halo.HostRows(x) for x in a]

    class H(object):
        pass
    hs = [H(), H()]
    hs[0].sends, hs[0].receives = [np.zeros(0, np.int32), np.array([0, 1], np.int32)], \
        [np.zeros(0, np.int32), np.array([2], np.int32)]
    hs[1].sends, hs[1].receives = [np.array([1], np.int32), np.zeros(0, np.int32)], \
        [np.array([1, 2], np.int32), np.zeros(0, np.int32)]
    ex = [halo.DatExchange(rows[r], hs[r], comms[r]) for r in range(2)]
    pending = [e.begin() for e in ex]
    for p in pending:
        p.wait()
    np.testing.assert_array_equal(a[0][2], [12.0, 13.0])          # rank 1's row 1
    np.testing.assert_array_equal(a[1][1:], [[0.0, 1.0], [2.0, 3.0]])   # rank 0's rows 0, 1
    # a wait before the peer sent is a protocol error, not a hang
    lone = halo.LocalGroup(2).comms()
    req = lone[0].exchange([], [(1, halo.HostBuffer(np.zeros(1)))])
    with pytest.raises(RuntimeError):
        req.wait()


@pytest.mark.parametrize("op,want", [("sum", 6.0), ("min", 1.0), ("max", 3.0)])
def test_local_allreduce(op, want):
    comms = halo.LocalGroup(3).comms()
    vals = [np.array([float(r + 1)]) for r in range(3)]
    reds = [halo.GlobalReduction(halo.HostBuffer(vals[r]), comms[r], op) for r in range(3)]
    started = [x.begin() for x in reds]
    for r in range(3):
        vals[r][0] += 100.0            # what the execute halo adds is dropped
    for s in started:
        s.wait()
    for v in vals:
        assert v[0] == want


def test_self_comm():
    c = halo.SelfComm()
    v = np.array([2.5])
    r = halo.GlobalReduction(halo.HostBuffer(v), c, "sum").begin()
    v[0] = 7.0
    r.wait()
    assert v[0] == 2.5
    with pytest.raises(RuntimeError):
        c.exchange([(1, halo.HostBuffer(v))], [])


class _FakeWork(object):
    def __init__(self, log):
        self.log = log

    def wait(self):
        self.log.append("wait")


class _FakeDist(object):
    """The parts of torch.distributed TorchComm calls, recording the order."""

    class ReduceOp(object):
        SUM, MIN, MAX = "sum", "min", "max"

    def __init__(self):
        self.log = []

    def isend(self, *a):
        pass

    irecv = isend

    def P2POp(self, op, tensor, peer, group, tag):
        return (op, tensor, peer)

    def batch_isend_irecv(self, ops):
        self.log.append("issue %d" % len(ops))
        return [_FakeWork(self.log)]

    def all_reduce(self, t, op, group, async_op):
        self.log.append("allreduce")
        return _FakeWork(self.log)


def test_torch_comm_holds_buffers_until_waited():
    # NCCL reads and writes the buffers on its own stream: the communicator
    # must keep them referenced until its wait has run
    import gc
    import weakref

    comm = halo.TorchComm.__new__(halo.TorchComm)
    comm.dist, comm.group, comm.stream = _FakeDist(), None, None
    comm.rank, comm.size, comm._nx = 0, 2, 0
    send, recv, red = (halo.HostBuffer(np.zeros(4)) for _ in range(3))
    refs = [weakref.ref(b) for b in (send, recv, red)]
    req = comm.exchange([(1, send)], [(1, recv)])
    rreq = comm.allreduce(red, "sum")
    del send, recv, red
    gc.collect()
    assert all(r() is not None for r in refs)
    req.wait()
    rreq.wait()
    gc.collect()
    assert all(r() is None for r in refs)
    assert comm.dist.log == ["issue 2", "allreduce", "wait", "wait"]


def test_loop_phase_order():
    seen = []

    class X(object):
        def __init__(self, name):
            self.name = name

        def begin(self):
            seen.append(self.name + " begin")
            return halo.Request(lambda: seen.append(self.name + " end"))
    launch = lambda a, b: seen.append("run %d-%d" % (a, b))  # noqa: E731
    halo.run(halo.loop_phases((2, 5, 7, 9), launch, [X("x")], [X("g")], exec_halo=True))
    assert seen == ["x begin", "run 0-2", "x end", "run 2-5", "g begin", "run 5-7", "g end"]
    seen.clear()
    # without a reduction the owned rest and the execute halo are one launch
    halo.run(halo.loop_phases((2, 5, 7, 9), launch, [X("x")], [], exec_halo=True))
    assert seen == ["x begin", "run 0-2", "x end", "run 2-7"]
    seen.clear()
    halo.run(halo.loop_phases((2, 5, 7, 9), launch, [X("x")], [X("g")], direct=True))
    assert seen == ["run 0-5", "g begin", "g end"]


# ------------------------------------------- airfoil split over ranks (oracle)
def _seq():
    sys.path.insert(0, ROOT)
    from oracle import seq
    return seq


def _oracle_consts(seq):
    """The airfoil Consts, declared once for every rank of the process."""
    for c in list(seq._CONSTS.values()):
        c.remove_from_namespace()
    seq.Const(1, airfoil.GAM, "gam", np.float64)
    seq.Const(1, airfoil.GM1, "gm1", np.float64)
    seq.Const(1, airfoil.CFL, "cfl", np.float64)
    seq.Const(1, airfoil.EPS, "eps", np.float64)
    seq.Const(4, airfoil.freestream(), "qinf", np.float64)


def _oracle_rank(seq, g, local, q0):
    """One rank's part of the airfoil problem on the oracle: sets of the
    rank's total size, its local Maps and rows."""
    S = local.sets
    o = airfoil.Airfoil()
    o.local = local
    tot = {k: S[k].sizes[3] for k in S}
    o.nodes, o.edges = seq.Set(tot["nodes"], 2), seq.Set(tot["edges"])
    o.bedges, o.cells, o.vcells = seq.Set(tot["bedges"]), seq.Set(tot["cells"]), seq.Set(tot["cells"], 4)
    lm = local.maps
    o.pedge = seq.Map(o.edges, o.nodes, 2, lm["pedge"][2])
    o.pecell = seq.Map(o.edges, o.cells, 2, lm["pecell"][2])
    o.pevcell = seq.Map(o.edges, o.vcells, 2, lm["pecell"][2])
    o.pbedge = seq.Map(o.bedges, o.nodes, 2, lm["pbedge"][2])
    o.pbecell = seq.Map(o.bedges, o.cells, 1, lm["pbecell"][2])
    o.pbevcell = seq.Map(o.bedges, o.vcells, 1, lm["pbecell"][2])
    o.pcell = seq.Map(o.cells, o.nodes, 4, lm["pcell"][2])
    o.p_bound = seq.Dat(o.bedges, S["bedges"].local_rows(np.asarray(g.p_bound).reshape(-1, 1)), np.int32)
    o.p_x = seq.Dat(o.nodes, S["nodes"].local_rows(np.asarray(g.x).reshape(-1, 2)))
    o.p_q = seq.Dat(o.vcells, S["cells"].local_rows(q0))
    o.p_qold = seq.Dat(o.vcells, S["cells"].local_rows(q0))
    o.p_adt = seq.Dat(o.cells, np.zeros(tot["cells"]))
    o.p_res = seq.Dat(o.vcells, np.zeros((tot["cells"], 4)))
    o.k_save = seq.Kernel(airfoil.SAVE_SOLN, "save_soln")
    o.k_adt = seq.Kernel(airfoil.ADT_CALC, "adt_calc")
    o.k_res = seq.Kernel(airfoil.RES_CALC, "res_calc")
    o.k_bres = seq.Kernel(airfoil.BRES_CALC, "bres_calc")
    o.k_update = seq.Kernel(airfoil.UPDATE, "update")
    o.set_of = {id(o.p_bound): "bedges", id(o.p_x): "nodes", id(o.p_q): "cells",
                id(o.p_qold): "cells", id(o.p_adt): "cells", id(o.p_res): "cells"}
    o.name_of = {id(o.nodes): "nodes", id(o.edges): "edges", id(o.bedges): "bedges",
                 id(o.cells): "cells", id(o.vcells): "cells"}
    return o


class _Recorder(object):
    """The oracle's op2 API with par_loop recorded instead of run."""

    def __init__(self, seq):
        self._seq, self.calls = seq, []

    def __getattr__(self, name):
        return getattr(self._seq, name)

    def par_loop(self, kernel, iterset, *args):
        self.calls.append((kernel, iterset, args))


def _oracle_phases(seq, o, comm, kernel, iterset, args):
    """A loop of rank ``o`` over its partitioned set: every Dat an indirect
    loop reads is exchanged (the host test does not track stale halos)."""
    ls = o.local.sets[o.name_of[id(iterset)]]
    indirect = [a for a in args if a.map is not None and a.map is not seq.IdentityMap]
    direct = not indirect
    ex, seen = [], set()
    if not direct:
        for a in args:
            if isinstance(a.data, seq.Dat) and a.access in (seq.READ, seq.RW) and id(a.data) not in seen:
                seen.add(id(a.data))
                ex.append(halo.DatExchange(halo.HostRows(a.data.data),
                                           o.local.sets[o.set_of[id(a.data)]], comm))
    red = [halo.GlobalReduction(halo.HostBuffer(a.data.data), comm, "sum")
           for a in args if isinstance(a.data, seq.Global) and a.access is seq.INC]
    exec_halo = any(a.access is not seq.READ for a in indirect)

    def launch(s, e):
        seq.par_loop(kernel, iterset, *args, span=(s, e))
    return halo.loop_phases(ls.sizes, launch, ex, red, direct, exec_halo)


def _reference_run(seq, g, q0, iters):
    for c in list(seq._CONSTS.values()):
        c.remove_from_namespace()
    O = airfoil.build(seq, 0, 0, grid=g, q0=q0.copy())
    rms = []
    for _ in range(iters):
        r = airfoil.iteration(seq, O)
        rms.append(float(r.data[0]))
    return O.p_q.data.copy(), rms


def _gather_q(g, parts, ranks):
    q = np.full((g.ncells, 4), np.nan)
    for local, o in zip(parts, ranks):
        ls = local.sets["cells"]
        q[ls.l2g[:ls.sizes[1]]] = o.p_q.data[:ls.sizes[1]]
    return q


@pytest.mark.parametrize("nranks", [2, 3])
def test_partitioned_airfoil_in_process_matches_oracle(nranks):
    seq = _seq()
    g = meshes.airfoil_grid(24, 12, 2)
    q0 = airfoil.initial_q(g.ncells, 2).reshape(-1, 4)
    ref_q, ref_rms = _reference_run(seq, g, q0, 3)
    parts = airfoil.partition_grid(g, nranks)
    comms = halo.LocalGroup(nranks).comms()
    _oracle_consts(seq)
    ranks = [_oracle_rank(seq, g, p, q0) for p in parts]
    rms = []
    for _ in range(3):
        recs = [_Recorder(seq) for _ in ranks]
        outs = [airfoil.iteration(rec, o) for rec, o in zip(recs, ranks)]
        for k in range(len(recs[0].calls)):
            halo.run_lockstep([_oracle_phases(seq, o, comms[r], *recs[r].calls[k])
                               for r, o in enumerate(ranks)])
        vals = [float(x.data[0]) for x in outs]
        assert max(vals) == min(vals)             # every rank holds the reduced value
        rms.append(vals[0])
    q = _gather_q(g, parts, ranks)
    assert np.abs(q - ref_q).max() <= TOL * np.abs(ref_q).max()
    for a, b in zip(rms, ref_rms):
        assert abs(a - b) <= TOL * abs(b)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _gloo_rank(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    try:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
        seq = _seq()
        g = meshes.airfoil_grid(24, 12, 2)
        q0 = airfoil.initial_q(g.ncells, 2).reshape(-1, 4)
        parts = airfoil.partition_grid(g, ws)
        comm = halo.TorchComm()
        _oracle_consts(seq)
        o = _oracle_rank(seq, g, parts[rank], q0)
        rms = []
        for _ in range(3):
            rec = _Recorder(seq)
            r = airfoil.iteration(rec, o)
            for call in rec.calls:
                halo.run(_oracle_phases(seq, o, comm, *call))
            rms.append(float(r.data[0]))
        ls = parts[rank].sets["cells"]
        out.put((rank, ls.l2g[:ls.sizes[1]].tolist(), o.p_q.data[:ls.sizes[1]].tolist(), rms))
        dist.destroy_process_group()
    except Exception as e:  # pragma: no cover - reported through the queue
        import traceback
        out.put((rank, "error", traceback.format_exc(), repr(e)))


def test_partitioned_airfoil_two_gloo_ranks_matches_oracle():
    seq = _seq()
    g = meshes.airfoil_grid(24, 12, 2)
    q0 = airfoil.initial_q(g.ncells, 2).reshape(-1, 4)
    ref_q, ref_rms = _reference_run(seq, g, q0, 3)
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_gloo_rank, args=(r, ws, port, out)) for r in range(ws)]
    for p in procs:
        p.start()
    res = [out.get(timeout=300) for _ in range(ws)]
    for p in procs:
        p.join(timeout=60)
    for r in res:
        assert r[1] != "error", r[2]
    q = np.full((g.ncells, 4), np.nan)
    for rank, ids, rows, rms in res:
        q[np.asarray(ids)] = np.asarray(rows)
        for a, b in zip(rms, ref_rms):
            assert abs(a - b) <= TOL * abs(b)
    assert np.abs(q - ref_q).max() <= TOL * np.abs(ref_q).max()
    for p in procs:
        assert p.exitcode == 0


def test_halo_declaration_checks():
    """op2.Halo takes the backend's communicator by default (one rank here)
    and checks its lists as the reference does (pyop2/base.py:424-447)."""
    from pyop2_b200 import _lib, backends, base
    if backends.get_backend() == "pyop2_b200.void":
        backends.set_backend("b200")
    _lib.load()
    h = base.Halo([[]], [[]])
    assert h.comm.size == 1 and h.comm.rank == 0
    with pytest.raises(AssertionError):
        base.Halo([[], []], [[]])                    # two sends on one rank
    with pytest.raises(AssertionError):
        base.Halo([[0]], [[]])                       # a self-send
    comms = halo.LocalGroup(2).comms()
    h1 = base.Halo([[1, 2], []], [[5], []], comm=comms[1])
    s = base.Set([2, 3, 4, 6], 1, "checked", halo=h1)
    assert s.halo is h1 and s.sizes == (2, 3, 4, 6)
    with pytest.raises(AssertionError):
        base.Set([2, 3, 4, 6], 1, "bad", halo=base.Halo([[3], []], [[5], []], comm=comms[1]))
