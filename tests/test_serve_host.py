"""Host logic of the serving engine (no GPU): the HBM budget store, the
trace generator and the mesh byte estimates."""

import numpy as np
import pytest

from pyop2_b200.serve import MeshStore, P1Mesh, QuadMesh
from pyop2_b200.workloads import serving
from pyop2_b200.workloads.meshes import airfoil_grid, rect_p1


class FakeMesh(object):
    def __init__(self, mid, nbytes):
        self.mid, self.nbytes, self.refs = mid, nbytes, 0


def _store(budget, sizes):
    s = MeshStore(budget)
    for mid, n in sizes.items():
        s.register(mid, lambda mid=mid, n=n: FakeMesh(mid, n), n)
    return s


def test_store_loads_within_budget_and_evicts_lru_idle_meshes():
    s = _store(100, {"a": 40, "b": 40, "c": 40})
    a, b = s.load("a"), s.load("b")
    assert s.used == 80
    a.refs = 1                       # a is in use: never evicted
    s.get("b")
    c = s.load("c")                  # evicts the idle LRU mesh: b
    assert c is not None and "b" not in s.meshes and "a" in s.meshes
    assert s.used == 80
    assert s.reserve(20) and s.used == 100
    assert s.reserve(1)              # the idle mesh c is evicted to make room
    assert "c" not in s.meshes and s.used == 61
    s.release(21)
    c = s.load("c")
    c.refs = 1
    assert s.load("b") is None       # both resident meshes in use: no room
    assert s.used == 80


def test_store_reserve_evicts_only_what_is_needed():
    s = _store(100, {"a": 30, "b": 30, "c": 30})
    for m in "abc":
        s.load(m)
    assert s.reserve(20)             # evicts a (LRU) only
    assert list(s.meshes) == ["b", "c"] and s.used == 80


def test_trace_is_seeded_poisson_and_mixed():
    pool = serving.mesh_pool(4, 4, seed=1)
    t1 = serving.trace(2000, 2000.0, pool, seed=9)
    t2 = serving.trace(2000, 2000.0, pool, seed=9)
    assert [(j.arrival, j.mesh_id, j.seed) for j in t1] == [(j.arrival, j.mesh_id, j.seed) for j in t2]
    arr = np.array([j.arrival for j in t1])
    assert arr[0] == 0.0 and np.all(np.diff(arr) >= 0)
    rate = (len(arr) - 1) / arr[-1]
    assert 1800 < rate < 2200
    kinds = [j.kind for j in t1]
    assert 0.4 < kinds.count("p1") / len(kinds) < 0.6
    assert all(pool[j.mesh_id][0] == j.kind for j in t1)
    c = serving.clone_trace(t1[:5], realtime=False)
    assert all(j.arrival == 0.0 and j.result is None for j in c)


@pytest.mark.parametrize("nx,ny", [(1, 1), (5, 3), (30, 7)])
def test_mesh_byte_estimates_are_exact(nx, ny):
    coords, elem = rect_p1(nx, ny, seed=2)
    pairs = {(a, b) for t in elem for a in t for b in t}
    n, e = len(coords), len(elem)
    assert P1Mesh.estimate(nx, ny) == P1Mesh.device_bytes(n, e, len(pairs))
    g = airfoil_grid(max(nx, 2), max(ny, 2), 0)
    assert QuadMesh.estimate(max(nx, 2), max(ny, 2)) == QuadMesh.device_bytes(
        g.ncells, g.nnodes, g.nedges, g.nbedges)


class _Event(object):
    def record(self):
        return self

    def query(self):
        return True

    def synchronize(self):
        pass


class _Batch(object):
    sizes = []

    def __init__(self, insts, **kw):
        _Batch.sizes.append(len(insts))
        self.launches = 1

    def launch(self, sync_host=True):
        pass


class _Mesh(FakeMesh):
    def __init__(self, mid, nbytes, rb):
        FakeMesh.__init__(self, mid, nbytes)
        self.rb = rb

    def request_bytes(self):
        return self.rb


def _fake_jobs(n, meshes, steps, seed):
    from pyop2_b200 import serve

    class J(serve.Job):
        kind = "x"

        def __init__(self, rid, mid, nsteps):
            serve.Job.__init__(self, rid, 0.0, mid, 0)
            self.n = nsteps

        def admit(self, mesh):
            self.steps = [[("p1_mass", object())]] * self.n

        def readback(self, pool):
            pass

        def deliver(self, pool, consumer):
            consumer(self, {"rid": self.rid})

    rng = np.random.default_rng(seed)
    return [J(r, meshes[int(rng.integers(len(meshes)))], int(rng.integers(*steps)))
            for r in range(n)]


@pytest.mark.parametrize("steps,slots", [((1, 2), 1), ((1, 11), 3), ((5, 6), 2)])
def test_engine_admission_and_completion_logic(monkeypatch, steps, slots):
    """The engine's control flow with the device replaced by fakes: every
    request completes, the budget holds, requests share steps, and a batch
    of requests that all finish together does not stall admission."""
    from pyop2_b200 import serve
    monkeypatch.setattr(serve, "BatchLoop", _Batch)
    monkeypatch.setattr(serve.b200, "Event", _Event)
    sizes = {"m%d" % i: 100 + 37 * i for i in range(5)}
    store = MeshStore(10 ** 9)
    for m, n in sizes.items():
        store.register(m, lambda m=m, n=n: _Mesh(m, n, 10 + n // 10), n)
    for m in sizes:
        store.load(m)
    jobs = _fake_jobs(40, sorted(sizes), steps, seed=slots)
    need = max(10 + sizes[j.mesh_id] // 10 for j in jobs)
    tight = MeshStore(store.used + slots * need)
    tight.meshes, tight.used, tight.factories = (type(store.meshes)(store.meshes), store.used,
                                                 store.factories)
    _Batch.sizes = []
    eng = serve.Engine(tight, max_admit=3)
    done = eng.run(jobs, realtime=False)
    assert sorted(int(j.result["rid"]) for j in done) == list(range(40))
    assert eng.peak_used <= tight.budget
    assert tight.used == sum(m.nbytes for m in tight.meshes.values())
    if slots > 1:
        assert max(_Batch.sizes) > 1


def _fake_engine_env(monkeypatch, budget_slots=100):
    from pyop2_b200 import serve
    monkeypatch.setattr(serve, "BatchLoop", _Batch)
    monkeypatch.setattr(serve.b200, "Event", _Event)
    sizes = {"m%d" % i: 100 + 37 * i for i in range(5)}
    store = MeshStore(10 ** 9)
    for m, n in sizes.items():
        store.register(m, lambda m=m, n=n: _Mesh(m, n, 10 + n // 10), n)
    for m in sizes:
        store.load(m)
    return serve, store, sorted(sizes)


def test_full_admission_queue_rejects(monkeypatch):
    """Requests arriving to a full admission queue are rejected, not queued;
    the others complete and summary() counts both."""
    serve, store, meshes = _fake_engine_env(monkeypatch)
    jobs = _fake_jobs(30, meshes, (3, 4), seed=1)
    eng = serve.Engine(store, max_admit=2, max_waiting=5)
    done = eng.run(jobs, realtime=False)
    st = [j.status for j in done]
    # all 30 arrive at once: 5 fit the queue, the other 25 are turned away
    assert len(done) == 30 and st.count("rejected") == 25 and st.count("done") == 5
    s = serve.summary(done, t_first=0.0)
    assert s["requests"] == 5 and s["rejected"] == 25
    assert store.used == sum(m.nbytes for m in store.meshes.values())


def test_cancelled_requests_leave_and_return_memory(monkeypatch):
    """Cancelled before arrival, while waiting, or between steps: the request
    leaves with status 'cancelled', no result, and its memory back."""
    serve, store, meshes = _fake_engine_env(monkeypatch)
    jobs = _fake_jobs(20, meshes, (6, 7), seed=2)
    jobs[0].cancelled = True                      # before it arrives

    def consumer(job, views):
        job.result = views
        for j in jobs[10:15]:                     # withdrawn while others run
            j.cancelled = True
    eng = serve.Engine(store, max_admit=4, consumer=consumer)
    done = eng.run(jobs, realtime=False)
    by = {j.rid: j for j in done}
    assert len(by) == 20 and by[0].status == "cancelled" and by[0].result is None
    assert all(by[r].status == "cancelled" and by[r].result is None for r in range(10, 15))
    assert sum(j.status == "done" for j in done) == 14
    assert store.used == sum(m.nbytes for m in store.meshes.values())
    assert all(m.refs == 0 for m in store.meshes.values())
