"""Synthetic meshes (plain numpy arrays; no op2 objects).

* :func:`square_p1`: unit square, n x n quads split into two triangles along
  the (i, j) -> (i+1, j+1) diagonal; node (i, j) has id i*(n+1)+j.  P1 mass
  sparsity nnz = 7n^2+6n+1.
* :func:`square_p2`: the same triangles with P2 dofs on the (2n+1)^2 lattice
  (vertices at even, edge midpoints at odd lattice points); vertices jittered
  by up to ``jitter`` of the cell size from a seeded generator, midpoints at
  the mean of their jittered end points (affine P2).  nnz = 46n^2+16n+1.
* :func:`airfoil_grid`: an nx x ny quad grid on [0, 2] x [0, 1] laid out for
  the airfoil finite-volume loops: interior edges with their two end nodes and
  the two cells either side, boundary edges with their end nodes and cell,
  cell->node maps; cell and node numbering randomly permuted from a seed.
  Edge end points are ordered so that (dy, -dx) with (dx, dy) = x1 - x2 points
  from the first cell to the second (interior) or out of the domain
  (boundary), which is the orientation the airfoil flux kernels assume.
"""

import numpy as np


def square_p1(n):
    """Returns coords [(n+1)^2, 2] f64, elem_node [2 n^2, 3] i32."""
    m = n + 1
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    v00 = (i * m + j).ravel()
    v10 = ((i + 1) * m + j).ravel()
    v11 = ((i + 1) * m + j + 1).ravel()
    v01 = (i * m + j + 1).ravel()
    t1 = np.stack([v00, v10, v11], axis=1)
    t2 = np.stack([v00, v11, v01], axis=1)
    elem = np.empty((2 * n * n, 3), dtype=np.int32)
    elem[0::2] = t1
    elem[1::2] = t2
    xi, yj = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
    coords = np.stack([xi.ravel() / n, yj.ravel() / n], axis=1).astype(np.float64)
    return coords, elem


def rect_p1(nx, ny, seed=None):
    """nx x ny quads of side h = 1 / max(nx, ny), each split into two
    triangles; node numbering randomly permuted from ``seed`` (None keeps
    the structured numbering).  Returns coords [(nx+1)(ny+1), 2] f64 and
    elem_node [2 nx ny, 3] i32 (counter-clockwise)."""
    mx, my = nx + 1, ny + 1
    h = 1.0 / max(nx, ny)
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    v00 = (i * my + j).ravel()
    v10 = ((i + 1) * my + j).ravel()
    v11 = ((i + 1) * my + j + 1).ravel()
    v01 = (i * my + j + 1).ravel()
    elem = np.empty((2 * nx * ny, 3), dtype=np.int64)
    elem[0::2] = np.stack([v00, v10, v11], axis=1)
    elem[1::2] = np.stack([v00, v11, v01], axis=1)
    xi, yj = np.meshgrid(np.arange(mx), np.arange(my), indexing="ij")
    coords = np.stack([xi.ravel() * h, yj.ravel() * h], axis=1).astype(np.float64)
    if seed is not None:
        perm = np.random.default_rng(seed).permutation(mx * my)
        new_coords = np.empty_like(coords)
        new_coords[perm] = coords
        coords, elem = new_coords, perm[elem]
    return coords, elem.astype(np.int32)


def square_p2(n, seed=0, jitter=0.1):
    """Returns coords [(2n+1)^2, 2] f64 and elem_dof [2 n^2, 6] i32 with the
    local order (v0, v1, v2, m12, m02, m01): vertices then the midpoint of the
    edge opposite each vertex."""
    L = 2 * n + 1
    rng = np.random.default_rng(seed)
    h = 1.0 / n
    vx, vy = np.meshgrid(np.arange(n + 1) * h, np.arange(n + 1) * h, indexing="ij")
    jx = rng.uniform(-jitter, jitter, size=vx.shape) * h
    jy = rng.uniform(-jitter, jitter, size=vy.shape) * h
    # keep the boundary on the boundary
    jx[0, :] = jx[-1, :] = 0.0
    jy[:, 0] = jy[:, -1] = 0.0
    vx = vx + jx
    vy = vy + jy
    X = np.zeros((L, L))
    Y = np.zeros((L, L))
    X[0::2, 0::2], Y[0::2, 0::2] = vx, vy
    X[1::2, 0::2] = 0.5 * (vx[:-1, :] + vx[1:, :])
    Y[1::2, 0::2] = 0.5 * (vy[:-1, :] + vy[1:, :])
    X[0::2, 1::2] = 0.5 * (vx[:, :-1] + vx[:, 1:])
    Y[0::2, 1::2] = 0.5 * (vy[:, :-1] + vy[:, 1:])
    X[1::2, 1::2] = 0.5 * (vx[:-1, :-1] + vx[1:, 1:])
    Y[1::2, 1::2] = 0.5 * (vy[:-1, :-1] + vy[1:, 1:])
    coords = np.stack([X.ravel(), Y.ravel()], axis=1)
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    I, J = 2 * i.ravel(), 2 * j.ravel()

    def nid(a, b):
        return a * L + b

    # triangle A: (I,J), (I+2,J), (I+2,J+2); triangle B: (I,J), (I+2,J+2), (I,J+2)
    A = np.stack([nid(I, J), nid(I + 2, J), nid(I + 2, J + 2),
                  nid(I + 2, J + 1), nid(I + 1, J + 1), nid(I + 1, J)], axis=1)
    B = np.stack([nid(I, J), nid(I + 2, J + 2), nid(I, J + 2),
                  nid(I + 1, J + 2), nid(I, J + 1), nid(I + 1, J + 1)], axis=1)
    elem = np.empty((2 * n * n, 6), dtype=np.int32)
    elem[0::2] = A
    elem[1::2] = B
    return coords, elem


class AirfoilGrid(object):
    pass


def airfoil_grid(nx, ny, seed=0, permute=True):
    """Quad grid for the airfoil loops; see the module docstring."""
    g = AirfoilGrid()
    h = 1.0 / ny
    nnx, nny = nx + 1, ny + 1
    rng = np.random.default_rng(seed)
    node_perm = rng.permutation(nnx * nny) if permute else np.arange(nnx * nny)
    cell_perm = rng.permutation(nx * ny) if permute else np.arange(nx * ny)

    def node(i, j):  # structured id -> permuted id
        return node_perm[i * nny + j]

    def cell(i, j):
        return cell_perm[i * ny + j]

    xi, yj = np.meshgrid(np.arange(nnx), np.arange(nny), indexing="ij")
    x = np.empty((nnx * nny, 2))
    x[node_perm[(xi * nny + yj).ravel()]] = np.stack([xi.ravel() * h, yj.ravel() * h], axis=1)
    ci, cj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    ci, cj = ci.ravel(), cj.ravel()
    pcell = np.empty((nx * ny, 4), dtype=np.int32)
    pcell[cell(ci, cj)] = np.stack([node(ci, cj), node(ci + 1, cj), node(ci + 1, cj + 1),
                                    node(ci, cj + 1)], axis=1)
    # interior edges, structured order: vertical edges (between (i-1,j) and
    # (i,j)) then horizontal edges (between (i,j-1) and (i,j))
    vi, vj = np.meshgrid(np.arange(1, nx), np.arange(ny), indexing="ij")
    vi, vj = vi.ravel(), vj.ravel()
    ve_nodes = np.stack([node(vi, vj + 1), node(vi, vj)], axis=1)
    ve_cells = np.stack([cell(vi - 1, vj), cell(vi, vj)], axis=1)
    hi, hj = np.meshgrid(np.arange(nx), np.arange(1, ny), indexing="ij")
    hi, hj = hi.ravel(), hj.ravel()
    he_nodes = np.stack([node(hi, hj), node(hi + 1, hj)], axis=1)
    he_cells = np.stack([cell(hi, hj - 1), cell(hi, hj)], axis=1)
    g.pedge = np.concatenate([ve_nodes, he_nodes]).astype(np.int32)
    g.pecell = np.concatenate([ve_cells, he_cells]).astype(np.int32)
    # boundary edges: bottom (wall), top, left, right
    bi = np.arange(nx)
    bj = np.arange(ny)
    bottom_n = np.stack([node(bi + 1, 0), node(bi, 0)], axis=1)
    bottom_c = cell(bi, 0)
    top_n = np.stack([node(bi, ny), node(bi + 1, ny)], axis=1)
    top_c = cell(bi, ny - 1)
    left_n = np.stack([node(0, bj), node(0, bj + 1)], axis=1)
    left_c = cell(0, bj)
    right_n = np.stack([node(nx, bj + 1), node(nx, bj)], axis=1)
    right_c = cell(nx - 1, bj)
    g.pbedge = np.concatenate([bottom_n, top_n, left_n, right_n]).astype(np.int32)
    g.pbecell = np.concatenate([bottom_c, top_c, left_c, right_c]).astype(np.int32).reshape(-1, 1)
    g.p_bound = np.concatenate([np.ones(nx), np.full(nx, 2), np.full(ny, 2),
                                np.full(ny, 2)]).astype(np.int32).reshape(-1, 1)
    g.x = x
    g.pcell = pcell
    g.nnodes, g.ncells = nnx * nny, nx * ny
    g.nedges, g.nbedges = len(g.pedge), len(g.pbedge)
    return g
