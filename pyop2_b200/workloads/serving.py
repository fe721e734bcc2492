"""Serving workload: a pool of meshes and a Poisson request trace.

* P1 assembly requests on triangle meshes of log-uniform size (default
  10^3 .. 10^6 triangles; structured grids of random aspect ratio, node
  numbering permuted);
* airfoil-style chains of ``iters`` iterations on quad meshes of log-uniform
  size (default 10^4 .. 10^6 cells; cell and node numbering permuted).

Requests pick a mesh of their kind uniformly from the pool; inter-arrival
times are exponential with mean 1 / rate.  Everything derives from one seed.
"""

import numpy as np

from . import airfoil
from .meshes import airfoil_grid, rect_p1


def mesh_pool(n_p1, n_quad, seed=0, p1_range=(1e3, 1e6), quad_range=(1e4, 1e6)):
    """{mesh id: (kind, nx, ny)}."""
    rng = np.random.default_rng(seed)
    pool = {}
    for m in range(n_p1):
        tri = np.exp(rng.uniform(np.log(p1_range[0]), np.log(p1_range[1])))
        r = np.exp(rng.uniform(np.log(0.25), np.log(4.0)))
        quads = max(1.0, tri / 2)
        nx = max(1, int(round(np.sqrt(quads * r))))
        ny = max(1, int(round(quads / nx)))
        pool["p1_%d" % m] = ("p1", nx, ny)
    for m in range(n_quad):
        cells = np.exp(rng.uniform(np.log(quad_range[0]), np.log(quad_range[1])))
        ny = max(2, int(round(np.sqrt(cells / 2))))
        pool["quad_%d" % m] = ("quad", 2 * ny, ny)
    return pool


def declare_consts(op2):
    """The airfoil constants, shared by every chain request."""
    return [op2.Const(1, airfoil.GAM, "gam", np.float64), op2.Const(1, airfoil.GM1, "gm1", np.float64),
            op2.Const(1, airfoil.CFL, "cfl", np.float64), op2.Const(1, airfoil.EPS, "eps", np.float64),
            op2.Const(4, airfoil.freestream(), "qinf", np.float64)]


def register(store, op2, pool, seed=0):
    """Register a factory per mesh with the serving MeshStore."""
    from pyop2_b200.serve import P1Mesh, QuadMesh
    for k, (mid, (kind, nx, ny)) in enumerate(sorted(pool.items())):
        s = seed * 7919 + k
        if kind == "p1":
            def make(mid=mid, nx=nx, ny=ny, s=s):
                coords, elem = rect_p1(nx, ny, seed=s)
                return P1Mesh(op2, mid, coords, elem)
            hint = P1Mesh.estimate(nx, ny)
        else:
            def make(mid=mid, nx=nx, ny=ny, s=s):
                return QuadMesh(op2, mid, airfoil_grid(nx, ny, s))
            hint = QuadMesh.estimate(nx, ny)
        store.register(mid, make, hint)


def trace(n, rate, pool, seed=0, iters=10, p1_fraction=0.5):
    """n requests with Poisson arrivals at ``rate`` per second."""
    from pyop2_b200.serve import AssemblyJob, ChainJob
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    t -= t[0]
    p1 = sorted(m for m, v in pool.items() if v[0] == "p1")
    quad = sorted(m for m, v in pool.items() if v[0] == "quad")
    jobs = []
    for r in range(n):
        s = int(rng.integers(0, 2 ** 31))
        if (not quad) or (p1 and rng.random() < p1_fraction):
            jobs.append(AssemblyJob(r, float(t[r]), p1[int(rng.integers(len(p1)))], s))
        else:
            jobs.append(ChainJob(r, float(t[r]), quad[int(rng.integers(len(quad)))], s, iters))
    return jobs


def clone_trace(jobs, realtime=True):
    """Fresh copies of the jobs (same ids, arrivals, meshes and seeds)."""
    out = []
    for j in jobs:
        c = object.__new__(type(j))
        c.__dict__.update({k: v for k, v in j.__dict__.items()
                           if k in ("rid", "arrival", "mesh_id", "seed", "iters")})
        c.t_admit = c.t_done = c.result = c.status = None
        c.stage = 0
        c.cancelled = False
        if not realtime:
            c.arrival = 0.0
        out.append(c)
    return out
