"""Batching workload: many independent uneven triangle meshes, each with P1
mass and stiffness Mat assembly and an FP64 RHS INC loop.

Mesh m has E_m elements drawn log-uniform in [2^8, 2^16]; it is a structured
nx x ny quad grid (two triangles per quad, nx * ny = E_m / 2) of aspect ratio
nx / ny drawn log-uniform in [1/8, 8], with its node numbering randomly
permuted -- all from one seed.
"""

import numpy as np

from . import fem
from .meshes import rect_p1


def mesh_shapes(nmesh, seed=0, emin=2 ** 8, emax=2 ** 16):
    """(nx, ny) per mesh."""
    rng = np.random.default_rng(seed)
    e = np.exp(rng.uniform(np.log(emin), np.log(emax), size=nmesh))
    r = np.exp(rng.uniform(np.log(1.0 / 8), np.log(8.0), size=nmesh))
    quads = np.maximum(1, np.rint(e / 2))
    nx = np.maximum(1, np.rint(np.sqrt(quads * r))).astype(np.int64)
    ny = np.maximum(1, np.rint(quads / nx)).astype(np.int64)
    return list(zip(nx.tolist(), ny.tolist()))


def build(op2, shapes, seed=0):
    """One P1 problem (mass + stiffness Mats on one Sparsity, RHS) per mesh."""
    out = []
    for m, (nx, ny) in enumerate(shapes):
        coords, elem = rect_p1(nx, ny, seed=seed * 1000003 + m)
        out.append(fem.build_p1(op2, 0, coords=coords, elem=elem, stiffness=True))
    return out


def instances(op2, problems):
    """LoopInstances of the three loops of every mesh: (mass, stiffness, rhs)."""
    from pyop2_b200.batch import LoopInstance
    mass, stiff, rhs = [], [], []
    for P in problems:
        rows = (P.elem_node[op2.i[0]], P.elem_node[op2.i[1]])
        mass.append(LoopInstance(P.k_mass, P.elements(3, 3), P.mat(rows, op2.INC),
                                 P.coords(P.elem_vnode, op2.READ)))
        stiff.append(LoopInstance(P.k_stiff, P.elements(3, 3), P.stiff(rows, op2.INC),
                                  P.coords(P.elem_vnode, op2.READ)))
        rhs.append(LoopInstance(P.k_rhs, P.elements(3), P.b(P.elem_node[op2.i[0]], op2.INC),
                                P.coords(P.elem_vnode, op2.READ), P.f(P.elem_node, op2.READ)))
    return mass, stiff, rhs


def plain(op2, P):
    """The three loops of one mesh through op2.par_loop (the per-loop form)."""
    fem.assemble_p1(op2, P)          # mass + RHS
    fem.assemble_p1_stiffness(op2, P)


def bytes_per_mesh(P):
    """Algorithmic bytes of the three loops of one mesh."""
    nnz = int(P.sparsity.nz)
    return (2 * fem.assembly_bytes(P.n_elem, 3, P.n_nodes, nnz)
            + fem.rhs_bytes(P.n_elem, P.n_nodes))
