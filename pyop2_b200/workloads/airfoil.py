"""Airfoil-style finite-volume loop chain (the OP2 airfoil demo's loops).

Kernels: the arithmetic of the OP2 airfoil demo (save_soln, adt_calc,
res_calc, bres_calc, update; loop structure pyop2/demo/airfoil.py:86-131)
written out for this package.  Constants: gamma 1.4, gamma-1 0.4, CFL 0.9,
dissipation eps 0.05, free stream rho 1, u 0.5, v 0, p 1.

:func:`build` declares the Sets/Maps/Dats/Consts through any module with the
op2 API (the B200 backend's ``op2`` or the oracle), and :func:`iteration`
runs one outer iteration: save_soln, then twice (adt_calc, res_calc,
bres_calc, update with the rms reduction).
"""

import numpy as np

from .meshes import airfoil_grid

GAM = 1.4
GM1 = 0.4
CFL = 0.9
EPS = 0.05
RHO_INF, U_INF, V_INF, P_INF = 1.0, 0.5, 0.0, 1.0

SAVE_SOLN = """
void save_soln(double *q, double *qold) {
  for (int k = 0; k < 4; k++) qold[k] = q[k];
}
"""

# area / timestep of a cell from its four corners and state
ADT_CALC = """
void adt_calc(double *x1, double *x2, double *x3, double *x4, double *q, double *adt) {
  double rinv = 1.0 / q[0];
  double u = rinv * q[1];
  double v = rinv * q[2];
  double c = sqrt(gam * gm1 * (rinv * q[3] - 0.5 * (u * u + v * v)));
  double ex, ey;
  ex = x2[0] - x1[0]; ey = x2[1] - x1[1];
  *adt = fabs(u * ey - v * ex) + c * sqrt(ex * ex + ey * ey);
  ex = x3[0] - x2[0]; ey = x3[1] - x2[1];
  *adt += fabs(u * ey - v * ex) + c * sqrt(ex * ex + ey * ey);
  ex = x4[0] - x3[0]; ey = x4[1] - x3[1];
  *adt += fabs(u * ey - v * ex) + c * sqrt(ex * ex + ey * ey);
  ex = x1[0] - x4[0]; ey = x1[1] - x4[1];
  *adt += fabs(u * ey - v * ex) + c * sqrt(ex * ex + ey * ey);
  *adt = (*adt) / cfl;
}
"""

# central flux plus scalar dissipation across an interior edge
RES_CALC = """
void res_calc(double *x1, double *x2, double *q1, double *q2,
              double *adt1, double *adt2, double *res1, double *res2) {
  double ex = x1[0] - x2[0];
  double ey = x1[1] - x2[1];
  double r1 = 1.0 / q1[0];
  double pr1 = gm1 * (q1[3] - 0.5 * r1 * (q1[1] * q1[1] + q1[2] * q1[2]));
  double vn1 = r1 * (q1[1] * ey - q1[2] * ex);
  double r2 = 1.0 / q2[0];
  double pr2 = gm1 * (q2[3] - 0.5 * r2 * (q2[1] * q2[1] + q2[2] * q2[2]));
  double vn2 = r2 * (q2[1] * ey - q2[2] * ex);
  double diss = 0.5 * ((*adt1) + (*adt2)) * eps;
  double fl;
  fl = 0.5 * (vn1 * q1[0] + vn2 * q2[0]) + diss * (q1[0] - q2[0]);
  res1[0] += fl; res2[0] -= fl;
  fl = 0.5 * (vn1 * q1[1] + pr1 * ey + vn2 * q2[1] + pr2 * ey) + diss * (q1[1] - q2[1]);
  res1[1] += fl; res2[1] -= fl;
  fl = 0.5 * (vn1 * q1[2] - pr1 * ex + vn2 * q2[2] - pr2 * ex) + diss * (q1[2] - q2[2]);
  res1[2] += fl; res2[2] -= fl;
  fl = 0.5 * (vn1 * (q1[3] + pr1) + vn2 * (q2[3] + pr2)) + diss * (q1[3] - q2[3]);
  res1[3] += fl; res2[3] -= fl;
}
"""

# wall (bound == 1: pressure only) or far-field boundary flux
BRES_CALC = """
void bres_calc(double *x1, double *x2, double *q1, double *adt1, double *res1, int *bound) {
  double ex = x1[0] - x2[0];
  double ey = x1[1] - x2[1];
  double r1 = 1.0 / q1[0];
  double pr1 = gm1 * (q1[3] - 0.5 * r1 * (q1[1] * q1[1] + q1[2] * q1[2]));
  if (*bound == 1) {
    res1[1] += pr1 * ey;
    res1[2] += -pr1 * ex;
  } else {
    double vn1 = r1 * (q1[1] * ey - q1[2] * ex);
    double r2 = 1.0 / qinf[0];
    double pr2 = gm1 * (qinf[3] - 0.5 * r2 * (qinf[1] * qinf[1] + qinf[2] * qinf[2]));
    double vn2 = r2 * (qinf[1] * ey - qinf[2] * ex);
    double diss = (*adt1) * eps;
    double fl;
    fl = 0.5 * (vn1 * q1[0] + vn2 * qinf[0]) + diss * (q1[0] - qinf[0]);
    res1[0] += fl;
    fl = 0.5 * (vn1 * q1[1] + pr1 * ey + vn2 * qinf[1] + pr2 * ey) + diss * (q1[1] - qinf[1]);
    res1[1] += fl;
    fl = 0.5 * (vn1 * q1[2] - pr1 * ex + vn2 * qinf[2] - pr2 * ex) + diss * (q1[2] - qinf[2]);
    res1[2] += fl;
    fl = 0.5 * (vn1 * (q1[3] + pr1) + vn2 * (qinf[3] + pr2)) + diss * (q1[3] - qinf[3]);
    res1[3] += fl;
  }
}
"""

# explicit update with the residual; accumulates the squared change
UPDATE = """
void update(double *qold, double *q, double *res, double *adt, double *rms) {
  double ainv = 1.0 / (*adt);
  for (int k = 0; k < 4; k++) {
    double dq = ainv * res[k];
    q[k] = qold[k] - dq;
    res[k] = 0.0;
    *rms += dq * dq;
  }
}
"""


def freestream():
    e = P_INF / GM1 + 0.5 * RHO_INF * (U_INF ** 2 + V_INF ** 2)
    return np.array([RHO_INF, RHO_INF * U_INF, RHO_INF * V_INF, e])


def initial_q(ncells, seed=0, noise=0.01):
    rng = np.random.default_rng(seed + 1)
    return freestream()[None, :] * (1.0 + rng.uniform(-noise, noise, size=(ncells, 4)))


class Airfoil(object):
    """The op2 objects of one airfoil problem."""


def build(op2, nx, ny, seed=0, grid=None, consts=True, q0=None, qold0=None, zeros=None):
    """Declare the airfoil problem through ``op2`` (B200 op2 or the oracle).
    ``q0``/``qold0``/``zeros`` optionally supply the host arrays (e.g. pinned
    memory) of q, qold and of the zero-initialised adt/res."""
    g = grid if grid is not None else airfoil_grid(nx, ny, seed)
    A = Airfoil()
    A.grid = g
    A.nodes = op2.Set(g.nnodes, 2, "nodes")
    A.edges = op2.Set(g.nedges, 1, "edges")
    A.bedges = op2.Set(g.nbedges, 1, "bedges")
    A.cells = op2.Set(g.ncells, 1, "cells")
    A.vcells = op2.Set(g.ncells, 4, "vcells")
    A.pedge = op2.Map(A.edges, A.nodes, 2, g.pedge, "pedge")
    A.pecell = op2.Map(A.edges, A.cells, 2, g.pecell, "pecell")
    A.pevcell = op2.Map(A.edges, A.vcells, 2, g.pecell, "pevcell")
    A.pbedge = op2.Map(A.bedges, A.nodes, 2, g.pbedge, "pbedge")
    A.pbecell = op2.Map(A.bedges, A.cells, 1, g.pbecell, "pbecell")
    A.pbevcell = op2.Map(A.bedges, A.vcells, 1, g.pbecell, "pbevcell")
    A.pcell = op2.Map(A.cells, A.nodes, 4, g.pcell, "pcell")
    A.p_bound = op2.Dat(A.bedges, g.p_bound, np.int32, "p_bound")
    A.p_x = op2.Dat(A.nodes, g.x, np.float64, "p_x")
    if q0 is None:
        q0 = initial_q(g.ncells, seed)
    A.p_q = op2.Dat(A.vcells, q0, np.float64, "p_q")
    A.p_qold = op2.Dat(A.vcells, q0.copy() if qold0 is None else qold0, np.float64, "p_qold")
    za, zr = zeros if zeros is not None else (np.zeros(g.ncells), np.zeros((g.ncells, 4)))
    A.p_adt = op2.Dat(A.cells, za, np.float64, "p_adt")
    A.p_res = op2.Dat(A.vcells, zr, np.float64, "p_res")
    if consts:
        A.consts = [op2.Const(1, GAM, "gam", np.float64), op2.Const(1, GM1, "gm1", np.float64),
                    op2.Const(1, CFL, "cfl", np.float64), op2.Const(1, EPS, "eps", np.float64),
                    op2.Const(4, freestream(), "qinf", np.float64)]
    A.k_save = op2.Kernel(SAVE_SOLN, "save_soln")
    A.k_adt = op2.Kernel(ADT_CALC, "adt_calc")
    A.k_res = op2.Kernel(RES_CALC, "res_calc")
    A.k_bres = op2.Kernel(BRES_CALC, "bres_calc")
    A.k_update = op2.Kernel(UPDATE, "update")
    return A


MACH, ALPHA = 0.4, 0.0


def hdf5_layout(g, q0=None, seed=0):
    """The datasets of an OP2 airfoil mesh file (the names, shapes and
    attributes pyop2/demo/airfoil.py:45-75 reads from ``new_grid.h5``) for
    the grid ``g``: name -> (array, attributes).  Written to a file with
    h5py's ``create_dataset`` (one dataset per entry, attributes set from the
    dict), it is a mesh file the demo's reader accepts."""
    q = initial_q(g.ncells, seed) if q0 is None else np.asarray(q0, dtype=np.float64)
    dbl, i32 = {"type": "double"}, {"type": "int"}
    one = lambda v: np.array([v])
    return {
        "nodes": (one(g.nnodes), {}), "edges": (one(g.nedges), {}),
        "bedges": (one(g.nbedges), {}), "cells": (one(g.ncells), {}),
        "pedge": (np.asarray(g.pedge, np.int32).reshape(-1, 2), {}),
        "pecell": (np.asarray(g.pecell, np.int32).reshape(-1, 2), {}),
        "pbedge": (np.asarray(g.pbedge, np.int32).reshape(-1, 2), {}),
        "pbecell": (np.asarray(g.pbecell, np.int32).reshape(-1, 1), {}),
        "pcell": (np.asarray(g.pcell, np.int32).reshape(-1, 4), {}),
        "p_bound": (np.asarray(g.p_bound, np.int32).reshape(-1, 1), i32),
        "p_x": (np.asarray(g.x, np.float64).reshape(-1, 2), dbl),
        "p_q": (q.reshape(-1, 4), dbl), "p_qold": (q.reshape(-1, 4).copy(), dbl),
        "p_adt": (np.zeros((g.ncells, 1)), dbl), "p_res": (np.zeros((g.ncells, 4)), dbl),
        "gam": (one(GAM), {}), "gm1": (one(GM1), {}), "cfl": (one(CFL), {}),
        "eps": (one(EPS), {}), "mach": (one(MACH), {}), "alpha": (one(ALPHA), {}),
        "qinf": (freestream(), {}),
    }


def build_from_hdf5(op2, f):
    """Declare the airfoil problem from an OP2 airfoil mesh file ``f`` (an
    h5py File, or any object with its interface), with the declarations of
    pyop2/demo/airfoil.py:45-75: Sets, Maps and Dats through ``fromhdf5``."""
    A = Airfoil()
    A.grid = None
    A.vnodes = A.nodes = op2.Set.fromhdf5(f, "nodes", dim=2)
    A.edges = op2.Set.fromhdf5(f, "edges")
    A.bedges = op2.Set.fromhdf5(f, "bedges")
    A.cells = op2.Set.fromhdf5(f, "cells")
    A.vcells = op2.Set.fromhdf5(f, "cells", dim=4)
    A.pedge = op2.Map.fromhdf5(A.edges, A.vnodes, f, "pedge")
    A.pecell = op2.Map.fromhdf5(A.edges, A.cells, f, "pecell")
    A.pevcell = op2.Map.fromhdf5(A.edges, A.vcells, f, "pecell")
    A.pbedge = op2.Map.fromhdf5(A.bedges, A.vnodes, f, "pbedge")
    A.pbecell = op2.Map.fromhdf5(A.bedges, A.cells, f, "pbecell")
    A.pbevcell = op2.Map.fromhdf5(A.bedges, A.vcells, f, "pbecell")
    A.pcell = op2.Map.fromhdf5(A.cells, A.vnodes, f, "pcell")
    A.p_bound = op2.Dat.fromhdf5(A.bedges, f, "p_bound")
    A.p_x = op2.Dat.fromhdf5(A.vnodes, f, "p_x")
    A.p_q = op2.Dat.fromhdf5(A.vcells, f, "p_q")
    A.p_qold = op2.Dat.fromhdf5(A.vcells, f, "p_qold")
    A.p_adt = op2.Dat.fromhdf5(A.cells, f, "p_adt")
    A.p_res = op2.Dat.fromhdf5(A.vcells, f, "p_res")
    A.consts = [op2.Const.fromhdf5(f, n) for n in ("gam", "gm1", "cfl", "eps", "mach", "alpha", "qinf")]
    A.k_save = op2.Kernel(SAVE_SOLN, "save_soln")
    A.k_adt = op2.Kernel(ADT_CALC, "adt_calc")
    A.k_res = op2.Kernel(RES_CALC, "res_calc")
    A.k_bres = op2.Kernel(BRES_CALC, "bres_calc")
    A.k_update = op2.Kernel(UPDATE, "update")
    return A


def partition_grid(g, nranks):
    """Owner-computes partition of the airfoil mesh ``g`` over ``nranks``
    ranks (:func:`pyop2_b200.partition.partition`): cells in bands of their
    centroid's x coordinate, each edge and boundary edge with the owner of
    its first cell, each node with the owner of the lowest-numbered cell
    that holds it."""
    from ..partition import partition
    pcell = np.asarray(g.pcell, np.int64).reshape(-1, 4)
    pecell = np.asarray(g.pecell, np.int64).reshape(-1, 2)
    pbecell = np.asarray(g.pbecell, np.int64).reshape(-1, 1)
    cx = np.asarray(g.x, np.float64).reshape(-1, 2)[pcell, 0].mean(axis=1)
    cuts = np.quantile(cx, np.arange(1, nranks) / nranks) if nranks > 1 else np.zeros(0)
    cell_owner = np.searchsorted(cuts, cx, side="right").astype(np.int64)
    first = np.full(g.nnodes, g.ncells, np.int64)
    np.minimum.at(first, pcell.ravel(), np.repeat(np.arange(g.ncells), 4))
    node_owner = cell_owner[np.minimum(first, g.ncells - 1)]
    sets = {"nodes": g.nnodes, "edges": g.nedges, "bedges": g.nbedges, "cells": g.ncells}
    maps = {"pedge": ("edges", "nodes", g.pedge), "pecell": ("edges", "cells", pecell),
            "pbedge": ("bedges", "nodes", g.pbedge), "pbecell": ("bedges", "cells", pbecell),
            "pcell": ("cells", "nodes", pcell)}
    owner = {"cells": cell_owner, "nodes": node_owner, "edges": cell_owner[pecell[:, 0]],
             "bedges": cell_owner[pbecell[:, 0]]}
    return partition(sets, maps, owner, nranks)


def build_partitioned(op2, g, local, comm, seed=0, q0=None, consts=True):
    """Declare one rank's part of the airfoil problem (``local``: that
    rank's :class:`pyop2_b200.partition.LocalMesh` of :func:`partition_grid`)
    with Sets of four sizes and Halos over ``comm``, as a distributed run of
    the demo declares them; Dats hold the rank's rows of the global initial
    state, halo rows included."""
    A = Airfoil()
    A.grid, A.local = g, local
    S = local.sets

    def mkset(name, dim):
        ls = S[name]
        return op2.Set(list(ls.sizes), dim, name,
                       halo=op2.Halo(ls.sends, ls.receives, comm=comm))
    A.nodes = mkset("nodes", 2)
    A.edges = mkset("edges", 1)
    A.bedges = mkset("bedges", 1)
    A.cells = mkset("cells", 1)
    A.vcells = mkset("cells", 4)
    lm = local.maps
    A.pedge = op2.Map(A.edges, A.nodes, 2, lm["pedge"][2], "pedge")
    A.pecell = op2.Map(A.edges, A.cells, 2, lm["pecell"][2], "pecell")
    A.pevcell = op2.Map(A.edges, A.vcells, 2, lm["pecell"][2], "pevcell")
    A.pbedge = op2.Map(A.bedges, A.nodes, 2, lm["pbedge"][2], "pbedge")
    A.pbecell = op2.Map(A.bedges, A.cells, 1, lm["pbecell"][2], "pbecell")
    A.pbevcell = op2.Map(A.bedges, A.vcells, 1, lm["pbecell"][2], "pbevcell")
    A.pcell = op2.Map(A.cells, A.nodes, 4, lm["pcell"][2], "pcell")
    q = (initial_q(g.ncells, seed) if q0 is None else np.asarray(q0, np.float64)).reshape(-1, 4)
    cells = S["cells"]
    A.p_bound = op2.Dat(A.bedges, S["bedges"].local_rows(np.asarray(g.p_bound).reshape(-1, 1)),
                        np.int32, "p_bound")
    A.p_x = op2.Dat(A.nodes, S["nodes"].local_rows(np.asarray(g.x).reshape(-1, 2)), np.float64,
                    "p_x")
    A.p_q = op2.Dat(A.vcells, cells.local_rows(q), np.float64, "p_q")
    A.p_qold = op2.Dat(A.vcells, cells.local_rows(q), np.float64, "p_qold")
    A.p_adt = op2.Dat(A.cells, np.zeros(cells.sizes[3]), np.float64, "p_adt")
    A.p_res = op2.Dat(A.vcells, np.zeros((cells.sizes[3], 4)), np.float64, "p_res")
    for d in (A.p_bound, A.p_x, A.p_q, A.p_qold, A.p_adt, A.p_res):
        d.needs_halo_update = False        # halo rows start as copies of the owners' rows
    if consts:
        A.consts = [op2.Const(1, GAM, "gam", np.float64), op2.Const(1, GM1, "gm1", np.float64),
                    op2.Const(1, CFL, "cfl", np.float64), op2.Const(1, EPS, "eps", np.float64),
                    op2.Const(4, freestream(), "qinf", np.float64)]
    A.k_save = op2.Kernel(SAVE_SOLN, "save_soln")
    A.k_adt = op2.Kernel(ADT_CALC, "adt_calc")
    A.k_res = op2.Kernel(RES_CALC, "res_calc")
    A.k_bres = op2.Kernel(BRES_CALC, "bres_calc")
    A.k_update = op2.Kernel(UPDATE, "update")
    return A


def save_soln(op2, A):
    op2.par_loop(A.k_save, A.cells, A.p_q(op2.IdentityMap, op2.READ),
                 A.p_qold(op2.IdentityMap, op2.WRITE))


def adt_calc(op2, A):
    op2.par_loop(A.k_adt, A.cells,
                 A.p_x(A.pcell[0], op2.READ), A.p_x(A.pcell[1], op2.READ),
                 A.p_x(A.pcell[2], op2.READ), A.p_x(A.pcell[3], op2.READ),
                 A.p_q(op2.IdentityMap, op2.READ), A.p_adt(op2.IdentityMap, op2.WRITE))


def res_calc(op2, A):
    op2.par_loop(A.k_res, A.edges,
                 A.p_x(A.pedge[0], op2.READ), A.p_x(A.pedge[1], op2.READ),
                 A.p_q(A.pevcell[0], op2.READ), A.p_q(A.pevcell[1], op2.READ),
                 A.p_adt(A.pecell[0], op2.READ), A.p_adt(A.pecell[1], op2.READ),
                 A.p_res(A.pevcell[0], op2.INC), A.p_res(A.pevcell[1], op2.INC))


def bres_calc(op2, A):
    op2.par_loop(A.k_bres, A.bedges,
                 A.p_x(A.pbedge[0], op2.READ), A.p_x(A.pbedge[1], op2.READ),
                 A.p_q(A.pbevcell[0], op2.READ), A.p_adt(A.pbecell[0], op2.READ),
                 A.p_res(A.pbevcell[0], op2.INC), A.p_bound(op2.IdentityMap, op2.READ))


def update(op2, A, rms):
    op2.par_loop(A.k_update, A.cells,
                 A.p_qold(op2.IdentityMap, op2.READ), A.p_q(op2.IdentityMap, op2.WRITE),
                 A.p_res(op2.IdentityMap, op2.RW), A.p_adt(op2.IdentityMap, op2.READ),
                 rms(op2.INC))


def iteration(op2, A, rms=None):
    """One outer iteration (pyop2/demo/airfoil.py:88-131); returns the rms
    Global of the second update."""
    save_soln(op2, A)
    for _ in range(2):
        adt_calc(op2, A)
        res_calc(op2, A)
        bres_calc(op2, A)
        g = rms if rms is not None else op2.Global(1, 0.0, np.float64, "rms")
        update(op2, A, g)
    return g


def bytes_per_iteration(ncells, nnodes, nedges, nbedges):
    """Algorithmic (compulsory) bytes of one outer iteration: every distinct
    Map and Dat of a loop touched once (x2 for read-modify-write), maps with
    identical values (pecell/pevcell, pbecell/pbevcell) counted once."""
    f8 = 8
    save = ncells * 4 * f8 * 2
    adt = ncells * 4 * 4 + nnodes * 2 * f8 + ncells * 4 * f8 + ncells * f8
    res = (nedges * 2 * 4 * 2 + nnodes * 2 * f8 + ncells * 4 * f8 + ncells * f8 +
           2 * ncells * 4 * f8)
    bres = nbedges * (2 * 4 + 4 + 2 * 2 * f8 + 4 * f8 + f8 + 2 * 4 * f8 + 4)
    upd = ncells * 4 * f8 * 2 + 2 * ncells * 4 * f8 + ncells * f8
    return {"save_soln": save, "adt_calc": adt, "res_calc": res, "bres_calc": bres,
            "update": upd, "iteration": save + 2 * (adt + res + bres + upd)}
