"""Serving: a continuous-batching request loop over device-resident meshes.

Requests name a resident mesh and carry a small parameter (a scale factor
drawn from the request's seed); their input field is made on the device from
the mesh's base field.  Two kinds are served:

* :class:`AssemblyJob` -- P1 mass Mat + RHS assembly on a triangle mesh (the
  mass2d_triangle form) for the source f = s * f_base: one step;
* :class:`ChainJob` -- an airfoil-style chain of ``iters`` iterations
  (adt_calc, res_calc, bres_calc, update with an rms reduction; the initial
  state q = qinf + s * (q_base - qinf), then save_soln, first) on a quad
  mesh: one step per iteration.

:class:`Engine` admits arrived requests in order while their device memory
fits the HBM budget: a mesh is loaded once and shared; each request gets one
device *arena* holding all its arrays, and its loops are the mesh's template
loop instances with the arena's addresses patched into their parameter
blocks (no op2 objects per request).  Step after step the engine gathers the
next step of EVERY admitted request into one batched launch per loop kind
(:class:`pyop2_b200.batch.BatchLoop`): requests that arrive while others run
join at the next step and share the launches of the requests in flight.
Results come back by asynchronous copies into pinned host memory; a request
completes when the event after its last copy has passed, its results are
handed to the consumer and its arena is freed.  At most ``max_inflight``
steps are queued on the device ahead of the host, and at most ``max_admit``
requests are admitted between two steps.

:class:`PlainServer` is the per-request drop-in baseline: requests in arrival
order, each through the op2 API (op2 objects, one par_loop at a time,
results read back synchronously).

No counterpart in the reference, which ran one par_loop at a time from the
host (pyop2/cuda.py:656-658).
"""

import collections
import time

import numpy as np

from . import b200
from .batch import BatchLoop, LoopInstance
from ._lib import call
from .workloads import airfoil, fem

# launch order of loop kinds inside one step (each request's loops of a step
# appear in its own dependency order)
STEP_ORDER = ("q_init", "save_soln", "adt_calc", "res_calc", "bres_calc", "update",
              "p1_src", "p1_mass", "p1_rhs")
DEFAULT_CONFIG = dict(block_size=256, elems_per_thread=2, min_blocks=0, ctas_per_sm=0)

P1_SRC = """
void p1_src(double *f, double *fb, double *s) { f[0] = s[0] * fb[0]; }
"""

Q_INIT = """
void q_init(double *q, double *qb, double *s) {
  for (int k = 0; k < 4; k++) q[k] = qinf[k] + (qb[k] - qinf[k]) * s[0];
}
"""


def _align(n, a=256):
    return (int(n) + a - 1) // a * a


def _layout(sizes):
    """Offsets of consecutive 256-byte aligned sub-arrays, and the total."""
    offs, o = [], 0
    for n in sizes:
        offs.append(o)
        o += _align(n)
    return offs, o


def request_scale(seed):
    """The parameter a request carries: a factor in [0.5, 2)."""
    return float(np.random.default_rng(seed).uniform(0.5, 2.0))


# --------------------------------------------------------------- pinned pool
class PinnedPool(object):
    """Reusable pinned host buffers in power-of-two size classes (page-locked
    allocation costs milliseconds; a served request must not pay it)."""

    def __init__(self):
        self.free = collections.defaultdict(list)

    @staticmethod
    def size_class(nbytes):
        return max(256, 1 << (int(nbytes) - 1).bit_length())

    def take(self, nbytes):
        cls = self.size_class(nbytes)
        lst = self.free[cls]
        return lst.pop() if lst else b200.pinned_empty((cls,), np.uint8)

    def give(self, buf):
        self.free[buf.nbytes].append(buf)

    def reserve(self, nbytes, count):
        """Pre-allocate ``count`` buffers of the class holding nbytes."""
        cls = self.size_class(nbytes)
        while len(self.free[cls]) < count:
            self.free[cls].append(b200.pinned_empty((cls,), np.uint8))


POOL = PinnedPool()


# ---------------------------------------------------------------- meshes
class Mesh(object):
    """A device-resident mesh: its op2 Sets, Maps and shared Dats, and per
    loop kind a template LoopInstance bound to placeholder objects that
    requests replace by their arena's addresses."""

    def __init__(self, mid, kind, nbytes):
        self.mid, self.kind, self.nbytes = mid, kind, nbytes
        self.refs = 0


class P1Mesh(Mesh):
    def __init__(self, op2, mid, coords, elem):
        P = fem.build_p1(op2, 0, coords=coords, elem=elem)
        self.P = P
        # placeholders of per-request data: P.mat, P.b, f_req, s
        self.f_req = op2.Dat(P.nodes, None, np.float64, "f_req")
        self.s = op2.Global(1, 1.0, np.float64, "s")
        self.k_src = op2.Kernel(P1_SRC, "p1_src")
        rows = (P.elem_node[op2.i[0]], P.elem_node[op2.i[1]])
        self.t_src = LoopInstance(self.k_src, P.nodes, self.f_req(op2.IdentityMap, op2.WRITE),
                                  P.f(op2.IdentityMap, op2.READ), self.s(op2.READ))
        self.t_mass = LoopInstance(P.k_mass, P.elements(3, 3), P.mat(rows, op2.INC),
                                   P.coords(P.elem_vnode, op2.READ))
        self.t_rhs = LoopInstance(P.k_rhs, P.elements(3), P.b(P.elem_node[op2.i[0]], op2.INC),
                                  P.coords(P.elem_vnode, op2.READ),
                                  self.f_req(P.elem_node, op2.READ))
        nnz = int(P.sparsity.nz)
        n, e = P.n_nodes, P.n_elem
        Mesh.__init__(self, mid, "p1", self.device_bytes(n, e, nnz))
        self.nnz, self.nodes, self.elements = nnz, n, e
        self.offs, self.arena_bytes = _layout([nnz * 8, n * 8, n * 8, 8])

    @staticmethod
    def device_bytes(n, e, nnz):
        """Map, coordinates, base field, CSR (rowptr, colidx, nnz), slot
        table and the placeholders' Mat values and Dats."""
        return (e * 3 * 4 + n * 16 + (n + 1) * 4 + nnz * 4 + n * 4 + e * 9 * 4
                + nnz * 8 + 4 * n * 8)

    @classmethod
    def estimate(cls, nx, ny):
        """device_bytes of an nx x ny two-triangles-per-quad grid."""
        n, e = (nx + 1) * (ny + 1), 2 * nx * ny
        return cls.device_bytes(n, e, 7 * nx * ny + 3 * (nx + ny) + 1)

    def request_bytes(self):
        return self.arena_bytes


class QuadMesh(Mesh):
    def __init__(self, op2, mid, grid):
        A = airfoil.build(op2, 0, 0, grid=grid, consts=False)
        self.A = A
        self.q_base = op2.Dat(A.vcells, airfoil.initial_q(grid.ncells, 1), np.float64, "q_base")
        self.s = op2.Global(1, 1.0, np.float64, "s")
        self.rms = op2.Global(1, 0.0, np.float64, "rms")
        self.k_init = op2.Kernel(Q_INIT, "q_init")
        self.t_init = LoopInstance(self.k_init, A.cells, A.p_q(op2.IdentityMap, op2.WRITE),
                                   self.q_base(op2.IdentityMap, op2.READ), self.s(op2.READ))
        self.t_save = LoopInstance(A.k_save, A.cells, A.p_q(op2.IdentityMap, op2.READ),
                                   A.p_qold(op2.IdentityMap, op2.WRITE))
        self.t_adt = LoopInstance(A.k_adt, A.cells,
                                  A.p_x(A.pcell[0], op2.READ), A.p_x(A.pcell[1], op2.READ),
                                  A.p_x(A.pcell[2], op2.READ), A.p_x(A.pcell[3], op2.READ),
                                  A.p_q(op2.IdentityMap, op2.READ),
                                  A.p_adt(op2.IdentityMap, op2.WRITE))
        self.t_res = LoopInstance(A.k_res, A.edges,
                                  A.p_x(A.pedge[0], op2.READ), A.p_x(A.pedge[1], op2.READ),
                                  A.p_q(A.pevcell[0], op2.READ), A.p_q(A.pevcell[1], op2.READ),
                                  A.p_adt(A.pecell[0], op2.READ), A.p_adt(A.pecell[1], op2.READ),
                                  A.p_res(A.pevcell[0], op2.INC), A.p_res(A.pevcell[1], op2.INC))
        self.t_bres = LoopInstance(A.k_bres, A.bedges,
                                   A.p_x(A.pbedge[0], op2.READ), A.p_x(A.pbedge[1], op2.READ),
                                   A.p_q(A.pbevcell[0], op2.READ), A.p_adt(A.pbecell[0], op2.READ),
                                   A.p_res(A.pbevcell[0], op2.INC),
                                   A.p_bound(op2.IdentityMap, op2.READ))
        self.t_update = LoopInstance(A.k_update, A.cells,
                                     A.p_qold(op2.IdentityMap, op2.READ),
                                     A.p_q(op2.IdentityMap, op2.WRITE),
                                     A.p_res(op2.IdentityMap, op2.RW),
                                     A.p_adt(op2.IdentityMap, op2.READ), self.rms(op2.INC))
        g = grid
        Mesh.__init__(self, mid, "quad", self.device_bytes(g.ncells, g.nnodes, g.nedges, g.nbedges))
        self.cells = g.ncells
        c = g.ncells
        self.offs, self.arena_bytes = _layout([c * 32, c * 32, c * 32, c * 8, 8, 8])

    @staticmethod
    def device_bytes(cells, nodes, edges, bedges):
        """Maps, node coordinates, boundary flags, the base state and the
        placeholders' Dats."""
        return edges * 16 + bedges * 12 + cells * 16 + nodes * 16 + bedges * 4 + cells * 136

    @classmethod
    def estimate(cls, nx, ny):
        return cls.device_bytes(nx * ny, (nx + 1) * (ny + 1), (nx - 1) * ny + nx * (ny - 1),
                                2 * (nx + ny))

    def request_bytes(self):
        return self.arena_bytes


# ----------------------------------------------------------------- requests
class Job(object):
    """One request: arrival time (s from the start of the trace), the mesh
    it names and its seed (which gives its scale parameter)."""

    kind = None

    def __init__(self, rid, arrival, mesh_id, seed):
        self.rid, self.arrival, self.mesh_id, self.seed = rid, arrival, mesh_id, seed
        self.t_admit = self.t_done = None
        self.result = None
        self.stage = 0
        # 'done', 'rejected' (admission queue full) or 'cancelled'; a caller
        # sets ``cancelled`` to withdraw the request (see Engine.run)
        self.status = None
        self.cancelled = False

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.arrival

    def _arena(self, mesh):
        self.arena = b200.DeviceBuffer(mesh.arena_bytes)
        self.arena.memset(0)
        s = np.array([request_scale(self.seed)])
        base = self.arena.ptr
        call("op2b_memcpy_h2d", base + mesh.offs[-1], s.ctypes.data, 8, 0)
        return [base + o for o in mesh.offs]

    def _copy_back(self, pool, parts):
        """Asynchronous copies of (device address, bytes) parts into pinned
        buffers."""
        self._bufs = []
        for ptr, n in parts:
            buf = pool.take(n)
            call("op2b_memcpy_d2h_async", buf.ctypes.data, ptr, n, 0)
            self._bufs.append((buf, n))

    def deliver(self, pool, consumer):
        views = [buf[:n] for buf, n in self._bufs]
        consumer(self, self._views(views))
        for buf, _ in self._bufs:
            pool.give(buf)
        self._bufs = None
        self.arena = None
        self.steps = None


class AssemblyJob(Job):
    kind = "p1"

    def admit(self, mesh):
        mat, b, f, s = self._arena(mesh)
        self._parts = [(mat, mesh.nnz * 8), (b, mesh.nodes * 8)]
        P = mesh.P
        self.steps = [[("p1_src", mesh.t_src.patch({mesh.f_req: f, mesh.s: s})),
                       ("p1_mass", mesh.t_mass.patch({P.mat: mat})),
                       ("p1_rhs", mesh.t_rhs.patch({P.b: b, mesh.f_req: f}))]]

    def readback(self, pool):
        self._copy_back(pool, self._parts)

    def _views(self, v):
        return {"mat": v[0].view(np.float64), "b": v[1].view(np.float64)}

    def run_plain(self, op2, mesh):
        """The per-request drop-in: op2 objects, one op2.par_loop at a time,
        synchronous reads."""
        P = mesh.P
        s = op2.Global(1, request_scale(self.seed), np.float64, "s")
        f = op2.Dat(P.nodes, None, np.float64, "f")
        b = op2.Dat(P.nodes, None, np.float64, "b")
        b.zero()
        mat = op2.Mat(P.sparsity, np.float64, "mass")
        mat.zero()
        op2.par_loop(mesh.k_src, P.nodes, f(op2.IdentityMap, op2.WRITE),
                     P.f(op2.IdentityMap, op2.READ), s(op2.READ))
        op2.par_loop(P.k_mass, P.elements(3, 3),
                     mat((P.elem_node[op2.i[0]], P.elem_node[op2.i[1]]), op2.INC),
                     P.coords(P.elem_vnode, op2.READ))
        op2.par_loop(P.k_rhs, P.elements(3), b(P.elem_node[op2.i[0]], op2.INC),
                     P.coords(P.elem_vnode, op2.READ), f(P.elem_node, op2.READ))
        return {"mat": mat.array, "b": b.data_ro.reshape(-1)}


class ChainJob(Job):
    kind = "quad"

    def __init__(self, rid, arrival, mesh_id, seed, iters=10):
        Job.__init__(self, rid, arrival, mesh_id, seed)
        self.iters = iters

    def admit(self, mesh):
        q, qold, res, adt, rms, s = self._arena(mesh)
        self._parts = [(q, mesh.cells * 32), (rms, 8)]
        A = mesh.A
        sub = {A.p_q: q, A.p_qold: qold, A.p_res: res, A.p_adt: adt, mesh.rms: rms}
        it = [("adt_calc", mesh.t_adt.patch(sub)), ("res_calc", mesh.t_res.patch(sub)),
              ("bres_calc", mesh.t_bres.patch(sub)), ("update", mesh.t_update.patch(sub))]
        first = [("q_init", mesh.t_init.patch({A.p_q: q, mesh.s: s})),
                 ("save_soln", mesh.t_save.patch(sub))]
        self.steps = [first + it] + [it] * (self.iters - 1)

    def readback(self, pool):
        self._copy_back(pool, self._parts)

    def _views(self, v):
        return {"q": v[0].view(np.float64).reshape(-1, 4), "rms": v[1].view(np.float64)}

    def run_plain(self, op2, mesh):
        A = mesh.A
        s = op2.Global(1, request_scale(self.seed), np.float64, "s")
        q = op2.Dat(A.vcells, None, np.float64, "q")
        qold = op2.Dat(A.vcells, None, np.float64, "qold")
        adt = op2.Dat(A.cells, None, np.float64, "adt")
        res = op2.Dat(A.vcells, None, np.float64, "res")
        res.zero()
        rms = op2.Global(1, 0.0, np.float64, "rms")
        op2.par_loop(mesh.k_init, A.cells, q(op2.IdentityMap, op2.WRITE),
                     mesh.q_base(op2.IdentityMap, op2.READ), s(op2.READ))
        op2.par_loop(A.k_save, A.cells, q(op2.IdentityMap, op2.READ),
                     qold(op2.IdentityMap, op2.WRITE))
        for _ in range(self.iters):
            op2.par_loop(A.k_adt, A.cells, A.p_x(A.pcell[0], op2.READ),
                         A.p_x(A.pcell[1], op2.READ), A.p_x(A.pcell[2], op2.READ),
                         A.p_x(A.pcell[3], op2.READ), q(op2.IdentityMap, op2.READ),
                         adt(op2.IdentityMap, op2.WRITE))
            op2.par_loop(A.k_res, A.edges, A.p_x(A.pedge[0], op2.READ),
                         A.p_x(A.pedge[1], op2.READ), q(A.pevcell[0], op2.READ),
                         q(A.pevcell[1], op2.READ), adt(A.pecell[0], op2.READ),
                         adt(A.pecell[1], op2.READ), res(A.pevcell[0], op2.INC),
                         res(A.pevcell[1], op2.INC))
            op2.par_loop(A.k_bres, A.bedges, A.p_x(A.pbedge[0], op2.READ),
                         A.p_x(A.pbedge[1], op2.READ), q(A.pbevcell[0], op2.READ),
                         adt(A.pbecell[0], op2.READ), res(A.pbevcell[0], op2.INC),
                         A.p_bound(op2.IdentityMap, op2.READ))
            op2.par_loop(A.k_update, A.cells, qold(op2.IdentityMap, op2.READ),
                         q(op2.IdentityMap, op2.WRITE), res(op2.IdentityMap, op2.RW),
                         adt(op2.IdentityMap, op2.READ), rms(op2.INC))
        return {"q": q.data_ro, "rms": rms.data_ro}


def keep_results(job, views):
    """Default consumer: keep a copy of the results on the job."""
    job.result = {k: np.array(v) for k, v in views.items()}


# ------------------------------------------------------------------- engine
class MeshStore(object):
    """Resident meshes against an HBM budget (bytes), LRU eviction of meshes
    no admitted request uses."""

    def __init__(self, budget=None):
        if budget is None:
            from . import configuration as cfg
            budget = float(cfg.cfg['hbm_budget_gb']) * 1e9
        self.budget = int(budget)
        self.used = 0
        self.meshes = collections.OrderedDict()
        self.factories = {}

    def register(self, mid, factory, nbytes_hint):
        self.factories[mid] = (factory, nbytes_hint)

    def reserve(self, nbytes):
        """Make room for nbytes by evicting idle meshes; False if it cannot."""
        if self.used + nbytes <= self.budget:
            self.used += nbytes
            return True
        for mid in list(self.meshes):
            if self.used + nbytes <= self.budget:
                break
            m = self.meshes[mid]
            if m.refs == 0:
                del self.meshes[mid]
                self.used -= m.nbytes
        if self.used + nbytes <= self.budget:
            self.used += nbytes
            return True
        return False

    def release(self, nbytes):
        self.used -= nbytes

    def get(self, mid):
        """The resident mesh, or None."""
        m = self.meshes.get(mid)
        if m is not None:
            self.meshes.move_to_end(mid)
        return m

    def load(self, mid):
        """Make mesh mid resident if the budget allows; returns it or None."""
        m = self.get(mid)
        if m is not None:
            return m
        factory, hint = self.factories[mid]
        if not self.reserve(hint):
            return None
        m = factory()
        self.used += m.nbytes - hint
        self.meshes[mid] = m
        return m


class Engine(object):
    """Continuous-batching server (see the module docstring).

    ``configs`` maps a loop kind to its BatchLoop configuration (e.g. from
    :mod:`pyop2_b200.autotune`); others use DEFAULT_CONFIG.  ``consumer(job,
    views)`` receives each completed request's results as views of pinned
    memory, valid during the call (default: :func:`keep_results`)."""

    def __init__(self, store, max_inflight=2, max_admit=64, configs=None, consumer=None,
                 pool=None, timing=False, max_waiting=None):
        self.store = store
        self.max_inflight, self.max_admit = max_inflight, max_admit
        # bound of the admission queue: a request arriving to a full queue is
        # rejected (status 'rejected') instead of waiting
        self.max_waiting = max_waiting
        self.configs = dict(configs or {})
        self.consumer = consumer or keep_results
        self.pool = pool if pool is not None else POOL
        self.steps = 0
        self.launches = 0
        self.batch_sizes = []
        self.peak_used = 0
        # with timing, a pair of events brackets every step's launches
        self.timing = timing
        self.step_events = []

    def gpu_busy_ms(self):
        """Device time of the steps' launches (timing=True), in ms."""
        return sum(a.elapsed_ms(b) for a, b in self.step_events)

    def run(self, jobs, realtime=True):
        """Serve ``jobs``.  Each is admitted no earlier than its arrival time
        (seconds from the start; ``realtime=False`` releases all at once).
        Returns the jobs in completion order with t_admit / t_done set."""
        pending = collections.deque(sorted(jobs, key=lambda j: j.arrival))
        waiting = collections.deque()
        active = []
        inflight = collections.deque()
        done = []
        t0 = time.perf_counter()
        clock = (lambda: time.perf_counter() - t0) if realtime else (lambda: float("inf"))
        while pending or waiting or active or inflight:
            now = clock()
            while pending and pending[0].arrival <= now:
                job = pending.popleft()
                if job.cancelled:
                    self._retire(job, "cancelled", t0, done)
                elif self.max_waiting is not None and len(waiting) >= self.max_waiting:
                    self._retire(job, "rejected", t0, done)
                else:
                    waiting.append(job)
            if any(j.cancelled for j in waiting):
                for j in [j for j in waiting if j.cancelled]:
                    self._retire(j, "cancelled", t0, done)
                waiting = collections.deque(j for j in waiting if not j.cancelled)
            # completions first: they return memory to the budget
            while inflight and inflight[0][0].query():
                self._complete(inflight.popleft()[1], t0, done)
            # admission, in arrival order, while memory allows
            admitted = 0
            while waiting and admitted < self.max_admit:
                job = waiting[0]
                mesh = self.store.load(job.mesh_id)
                if mesh is None:
                    break
                mesh.refs += 1          # not evictable while a request uses it
                if not self.store.reserve(mesh.request_bytes()):
                    mesh.refs -= 1
                    break
                waiting.popleft()
                job._mesh = mesh
                job.admit(mesh)
                job.t_admit = time.perf_counter() - t0
                active.append(job)
                admitted += 1
            self.peak_used = max(self.peak_used, self.store.used)
            if any(j.cancelled for j in active):
                # withdrawn between steps: its launched work completes in
                # stream order before the arena's stream-ordered free
                for j in [j for j in active if j.cancelled]:
                    j._mesh.refs -= 1
                    self.store.release(j._mesh.request_bytes())
                    j._mesh = j.arena = j.steps = None
                    self._retire(j, "cancelled", t0, done)
                active = [j for j in active if not j.cancelled]
            if active and len(inflight) < self.max_inflight:
                finishing = self._step(active)
                ev = b200.Event().record()
                inflight.append((ev, finishing))
                active = [j for j in active if j.stage < len(j.steps)]
            elif inflight:
                # the device is ahead: wait for the oldest step
                ev, fin = inflight.popleft()
                ev.synchronize()
                self._complete(fin, t0, done)
            elif pending and not waiting:
                wait = pending[0].arrival - clock()
                if wait > 0:
                    time.sleep(min(wait, 0.001))
            elif waiting and not active:
                raise RuntimeError("request %d (mesh %r) does not fit the HBM budget: %d of %d "
                                   "bytes in use by resident meshes" % (
                                       waiting[0].rid, waiting[0].mesh_id, self.store.used,
                                       self.store.budget))
        return done

    def _step(self, active):
        groups = collections.defaultdict(list)
        for job in active:
            for kind, inst in job.steps[job.stage]:
                groups[kind].append(inst)
        if self.timing:
            e0 = b200.Event().record()
        for kind in STEP_ORDER:
            insts = groups.get(kind)
            if not insts:
                continue
            bl = BatchLoop(insts, **self.configs.get(kind, DEFAULT_CONFIG))
            bl.launch(sync_host=False)
            self.launches += bl.launches
            self.batch_sizes.append(len(insts))
        if self.timing:
            self.step_events.append((e0, b200.Event().record()))
        finishing = []
        for job in active:
            job.stage += 1
            if job.stage == len(job.steps):
                job.readback(self.pool)
                finishing.append(job)
        self.steps += 1
        return finishing

    def _complete(self, jobs, t0, done):
        t = time.perf_counter() - t0
        for job in jobs:
            job.t_done = t
            job.status = "done"
            job.deliver(self.pool, self.consumer)
            job._mesh.refs -= 1
            self.store.release(job._mesh.request_bytes())
            job._mesh = None
            done.append(job)

    @staticmethod
    def _retire(job, status, t0, done):
        """A request that leaves without a result (rejected or cancelled)."""
        job.status = status
        job.t_done = time.perf_counter() - t0
        done.append(job)


class PlainServer(object):
    """Per-request drop-in: each request in arrival order through the op2 API,
    results read back synchronously before the next request starts."""

    def __init__(self, op2, store, consumer=None):
        self.op2, self.store = op2, store
        self.consumer = consumer or keep_results

    def run(self, jobs, realtime=True):
        t0 = time.perf_counter()
        done = []
        for job in sorted(jobs, key=lambda j: j.arrival):
            if realtime:
                wait = job.arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
            mesh = self.store.load(job.mesh_id)
            if mesh is None:
                raise RuntimeError("mesh %r does not fit the HBM budget" % job.mesh_id)
            job.t_admit = time.perf_counter() - t0
            views = job.run_plain(self.op2, mesh)
            job.t_done = time.perf_counter() - t0
            job.status = "done"
            self.consumer(job, views)
            done.append(job)
        return done


def summary(jobs, t_first=None):
    """p50 / p99 latency (ms) and requests/s of the completed requests of a
    served trace, with the counts of rejected and cancelled ones."""
    dropped = collections.Counter(j.status for j in jobs if j.status not in (None, "done"))
    jobs = [j for j in jobs if j.status in (None, "done")]
    lat = np.array([j.latency for j in jobs]) * 1e3
    t_first = min(j.arrival for j in jobs) if t_first is None else t_first
    span = max(j.t_done for j in jobs) - t_first
    out = {"requests": len(jobs), "req_per_s": round(len(jobs) / span, 1),
           "rejected": dropped.get("rejected", 0), "cancelled": dropped.get("cancelled", 0),
           "p50_ms": round(float(np.percentile(lat, 50)), 3),
           "p99_ms": round(float(np.percentile(lat, 99)), 3),
           "mean_ms": round(float(lat.mean()), 3), "span_s": round(span, 4)}
    for kind in sorted({j.kind for j in jobs}):
        lk = np.array([j.latency for j in jobs if j.kind == kind]) * 1e3
        out["p50_ms_" + kind] = round(float(np.percentile(lk, 50)), 3)
        out["p99_ms_" + kind] = round(float(np.percentile(lk, 99)), 3)
    return out
