"""Serving on the GPU: the continuous-batching engine against the plain
per-request drop-in and against each request served alone.

Tolerances: P1 assembly results within 1e-12 normwise relative (atomic INC
order differs between batches); airfoil chains (10 iterations, the
res_calc INC order differs) within 1e-11 for q and rms."""

import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture
def served(backend):
    """A small mesh pool, resident, with the airfoil constants declared."""
    from pyop2_b200 import base, op2, serve
    from pyop2_b200.workloads import serving
    for c in list(base.Const._defs):
        c.remove_from_namespace()
    consts = serving.declare_consts(op2)
    pool = serving.mesh_pool(4, 3, seed=11, p1_range=(300, 20000), quad_range=(500, 20000))
    store = serve.MeshStore(budget=8 << 30)
    serving.register(store, op2, pool, seed=11)
    for mid in pool:
        store.load(mid)
    yield op2, store, pool
    del consts
    for c in list(base.Const._defs):
        c.remove_from_namespace()


def _compare(a, b):
    if "mat" in a.result:
        assert rel_err(a.result["mat"], b.result["mat"]) < 1e-12
        assert rel_err(a.result["b"], b.result["b"]) < 1e-12
    else:
        assert rel_err(a.result["q"], b.result["q"]) < 1e-11
        assert abs(a.result["rms"] - b.result["rms"]) <= 1e-11 * abs(b.result["rms"])


def test_engine_matches_plain_and_alone(served):
    from pyop2_b200 import serve
    from pyop2_b200.workloads import serving
    op2, store, pool = served
    jobs = serving.trace(40, 5000.0, pool, seed=3, iters=10)
    eng = serve.Engine(store, max_inflight=2)
    done = eng.run(serving.clone_trace(jobs, realtime=False), realtime=False)
    assert len(done) == len(jobs) and all(j.result is not None for j in done)
    assert max(eng.batch_sizes) > 1            # requests shared launches
    by_id = {j.rid: j for j in done}
    plain = serve.PlainServer(op2, store).run(serving.clone_trace(jobs, realtime=False),
                                              realtime=False)
    for p in plain:
        _compare(by_id[p.rid], p)
    # each of a few requests served alone gives the result it had in the mix
    for rid in (0, 7, 21, 39):
        alone = serve.Engine(store).run(serving.clone_trace([jobs[rid]], realtime=False),
                                             realtime=False)
        _compare(by_id[rid], alone[0])
    s = serve.summary(done, t_first=0.0)
    assert s["requests"] == 40 and s["p99_ms"] >= s["p50_ms"] > 0


def test_assembly_result_matches_oracle(served):
    """An assembly request's Mat and RHS against the sequential oracle."""
    from oracle import seq
    from pyop2_b200 import serve
    from pyop2_b200.workloads import fem, serving
    op2, store, pool = served
    jobs = [j for j in serving.trace(12, 1000.0, pool, seed=4) if j.kind == "p1"][:2]
    done = serve.Engine(store).run(serving.clone_trace(jobs, realtime=False), realtime=False)
    for j in done:
        mesh = store.get(j.mesh_id)
        P = mesh.P
        coords = P.coords.data_ro
        elem = P.elem_node.values
        Q = fem.build_p1(seq, 0, coords=coords, elem=elem)
        Q.f.data[:] = serve.request_scale(j.seed) * P.f.data_ro.reshape(Q.f.data.shape)
        fem.assemble_p1(seq, Q)
        assert rel_err(j.result["mat"], Q.mat.array) < 1e-12
        assert rel_err(j.result["b"], Q.b.data.reshape(-1)) < 1e-12


def test_admission_respects_budget(served):
    """With a budget that holds the meshes and only a few requests at a time,
    requests wait for memory, all complete, and the budget is never
    exceeded."""
    from pyop2_b200 import serve
    from pyop2_b200.workloads import serving
    op2, store, pool = served
    jobs = serving.trace(30, 1e6, pool, seed=5)
    need = max(store.get(j.mesh_id).request_bytes() for j in jobs)
    tight = serve.MeshStore(budget=store.used + 3 * need)
    tight.meshes, tight.used, tight.factories = (type(store.meshes)(store.meshes), store.used,
                                                 store.factories)
    eng = serve.Engine(tight, max_inflight=2, max_admit=4)
    done = eng.run(serving.clone_trace(jobs, realtime=False), realtime=False)
    assert len(done) == 30
    assert eng.peak_used <= tight.budget
    # every request's memory returned: only resident meshes remain counted
    assert tight.used == sum(m.nbytes for m in tight.meshes.values())
    assert eng.steps > 10                      # admitted in waves, not all at once


def test_request_too_large_for_budget_raises(served):
    from pyop2_b200 import serve
    from pyop2_b200.workloads import serving
    op2, store, pool = served
    jobs = serving.trace(3, 1e6, pool, seed=6)
    tiny = serve.MeshStore(budget=1000)         # no mesh fits
    tiny.factories = store.factories
    with pytest.raises(RuntimeError):
        serve.Engine(tiny).run(serving.clone_trace(jobs, realtime=False), realtime=False)
