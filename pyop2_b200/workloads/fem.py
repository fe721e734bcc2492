"""Finite-element assembly workloads (P1 mass + RHS, P2 stiffness + mass).

Kernels are written for this package in the form the reference's FFC
kernels take (pyop2 test/unit/test_matrices.py:273-377): one local matrix
entry per call through a 2-d iteration space, coordinates through a vec-map.

* P1: mass matrix with the 3-point rule (basis values 2/3, 1/6,
  weights 1/6), RHS of f at the same points.
* P2: quadratic Lagrange basis, local order (v0, v1, v2, m12, m02,
  m01); stiffness with the degree-2 three-point rule (exact for products of
  linear gradients), mass with Dunavant's degree-4 six-point rule.  The FP64
  kernels compute in double; the precision form computes in float on float
  coordinates and returns the entry as double, to be accumulated into an FP64
  Mat (Kahan-compensated in owner-computes mode).

:func:`build_p1` / :func:`build_p2` declare the problem through any op2-shaped
module (the B200 op2 or the oracle) and return the objects and the loops.
"""

import numpy as np

from .meshes import square_p1, square_p2

P1_MASS = """
void p1_mass(double A[1][1], double *x[2], int j, int k) {
  double a00 = x[1][0] - x[0][0], a01 = x[2][0] - x[0][0];
  double a10 = x[1][1] - x[0][1], a11 = x[2][1] - x[0][1];
  double area = fabs(a00 * a11 - a01 * a10);
  const double w = 1.0 / 6.0;
  const double phi[3][3] = {{2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0},
                            {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0},
                            {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0}};
  for (int q = 0; q < 3; q++) A[0][0] += phi[q][j] * phi[q][k] * w * area;
}
"""

P1_RHS = """
void p1_rhs(double *b, double *x[2], double **f, int j) {
  double a00 = x[1][0] - x[0][0], a01 = x[2][0] - x[0][0];
  double a10 = x[1][1] - x[0][1], a11 = x[2][1] - x[0][1];
  double area = fabs(a00 * a11 - a01 * a10);
  const double w = 1.0 / 6.0;
  const double phi[3][3] = {{2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0},
                            {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0},
                            {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0}};
  for (int q = 0; q < 3; q++) {
    double fq = 0.0;
    for (int r = 0; r < 3; r++) fq += phi[q][r] * f[r][0];
    b[0] += phi[q][j] * fq * w * area;
  }
}
"""

# P2 basis on the reference triangle with barycentrics l0 = 1-s-t, l1 = s,
# l2 = t: vertices li(2li-1), midpoints 4 la lb.  REAL is double or float.
P1_STIFF = """
void p1_stiff(double A[1][1], double *x[2], int j, int k) {
  double a00 = x[1][0] - x[0][0], a01 = x[2][0] - x[0][0];
  double a10 = x[1][1] - x[0][1], a11 = x[2][1] - x[0][1];
  double det = a00 * a11 - a01 * a10;
  const double rg[3][2] = {{-1.0, -1.0}, {1.0, 0.0}, {0.0, 1.0}};
  double gj0 = (a11 * rg[j][0] - a10 * rg[j][1]) / det;
  double gj1 = (a00 * rg[j][1] - a01 * rg[j][0]) / det;
  double gk0 = (a11 * rg[k][0] - a10 * rg[k][1]) / det;
  double gk1 = (a00 * rg[k][1] - a01 * rg[k][0]) / det;
  A[0][0] += 0.5 * fabs(det) * (gj0 * gk0 + gj1 * gk1);
}
"""

_P2_COMMON = """
static __inline__ void p2_basis_%(S)s(REAL s, REAL t, REAL phi[6], REAL ds[6], REAL dt[6]) {
  const REAL l0 = (REAL)1 - s - t, l1 = s, l2 = t;
  phi[0] = l0 * ((REAL)2 * l0 - (REAL)1);
  phi[1] = l1 * ((REAL)2 * l1 - (REAL)1);
  phi[2] = l2 * ((REAL)2 * l2 - (REAL)1);
  phi[3] = (REAL)4 * l1 * l2;
  phi[4] = (REAL)4 * l0 * l2;
  phi[5] = (REAL)4 * l0 * l1;
  /* d/ds: dl0 = -1, dl1 = 1, dl2 = 0 ; d/dt: dl0 = -1, dl1 = 0, dl2 = 1 */
  ds[0] = -((REAL)4 * l0 - (REAL)1); dt[0] = ds[0];
  ds[1] = (REAL)4 * l1 - (REAL)1;    dt[1] = (REAL)0;
  ds[2] = (REAL)0;                   dt[2] = (REAL)4 * l2 - (REAL)1;
  ds[3] = (REAL)4 * l2;              dt[3] = (REAL)4 * l1;
  ds[4] = -(REAL)4 * l2;             dt[4] = (REAL)4 * (l0 - l2);
  ds[5] = (REAL)4 * (l0 - l1);       dt[5] = -(REAL)4 * l1;
}
"""

_P2_STIFF = """
void %(name)s(double A[1][1], %(X)s *x[2], int j, int k) {
  const REAL j00 = (REAL)(x[1][0] - x[0][0]), j01 = (REAL)(x[2][0] - x[0][0]);
  const REAL j10 = (REAL)(x[1][1] - x[0][1]), j11 = (REAL)(x[2][1] - x[0][1]);
  const REAL det = j00 * j11 - j01 * j10;
  const REAL inv = (REAL)1 / det;
  /* inverse Jacobian: grad_x = J^-T grad_ref */
  const REAL i00 = j11 * inv, i01 = -j01 * inv, i10 = -j10 * inv, i11 = j00 * inv;
  const REAL qs[3] = {(REAL)(1.0 / 6.0), (REAL)(2.0 / 3.0), (REAL)(1.0 / 6.0)};
  const REAL qt[3] = {(REAL)(1.0 / 6.0), (REAL)(1.0 / 6.0), (REAL)(2.0 / 3.0)};
  const REAL w = (REAL)(1.0 / 6.0);
  REAL sum = (REAL)0;
  for (int q = 0; q < 3; q++) {
    REAL phi[6], ds[6], dt[6];
    p2_basis_%(S)s(qs[q], qt[q], phi, ds, dt);
    const REAL gjx = i00 * ds[j] + i10 * dt[j], gjy = i01 * ds[j] + i11 * dt[j];
    const REAL gkx = i00 * ds[k] + i10 * dt[k], gky = i01 * ds[k] + i11 * dt[k];
    sum += (gjx * gkx + gjy * gky) * w;
  }
  A[0][0] += (double)(sum * (det < (REAL)0 ? -det : det));
}
"""

_P2_MASS = """
void %(name)s(double A[1][1], %(X)s *x[2], int j, int k) {
  const REAL j00 = (REAL)(x[1][0] - x[0][0]), j01 = (REAL)(x[2][0] - x[0][0]);
  const REAL j10 = (REAL)(x[1][1] - x[0][1]), j11 = (REAL)(x[2][1] - x[0][1]);
  const REAL det = j00 * j11 - j01 * j10;
  const REAL a = (REAL)0.445948490915965, b = (REAL)0.091576213509771;
  const REAL wa = (REAL)(0.223381589678011 / 2.0), wb = (REAL)(0.109951743655322 / 2.0);
  const REAL qs[6] = {a, (REAL)1 - (REAL)2 * a, a, b, (REAL)1 - (REAL)2 * b, b};
  const REAL qt[6] = {a, a, (REAL)1 - (REAL)2 * a, b, b, (REAL)1 - (REAL)2 * b};
  const REAL qw[6] = {wa, wa, wa, wb, wb, wb};
  REAL sum = (REAL)0;
  for (int q = 0; q < 6; q++) {
    REAL phi[6], ds[6], dt[6];
    p2_basis_%(S)s(qs[q], qt[q], phi, ds, dt);
    sum += phi[j] * phi[k] * qw[q];
  }
  A[0][0] += (double)(sum * (det < (REAL)0 ? -det : det));
}
"""


def p2_kernels(precision="f64"):
    """(stiffness code, name), (mass code, name) for precision 'f64' (double
    math), 'f32' (float math, double coordinates: the Jacobian's coordinate
    differences are taken in double) or 'f32g' (float math on float
    coordinates; the differences of O(h) of O(1) coordinates then lose about
    log2(1/h) bits)."""
    real, xt, suffix = {"f64": ("double", "double", "f64"), "f32": ("float", "double", "f32"),
                        "f32g": ("float", "float", "f32g")}[precision]
    head = "#define REAL %s\n" % real + (_P2_COMMON % {"S": suffix}).replace("static __inline__ ", "static inline ")
    stiff = head + _P2_STIFF % {"name": "p2_stiffness_" + suffix, "X": xt, "S": suffix} + "#undef REAL\n"
    mass = head + _P2_MASS % {"name": "p2_mass_" + suffix, "X": xt, "S": suffix} + "#undef REAL\n"
    return (stiff, "p2_stiffness_" + suffix), (mass, "p2_mass_" + suffix)


def p2_km_kernel(precision="f64"):
    """(code, name) of ONE kernel computing the stiffness entry into A and
    the mass entry into M of local position (j, k): the two Mats of the P2
    workload assembled by one par_loop, so the map, the coordinates and the
    scatter positions are read once for both.  Each entry is computed by the
    same arithmetic as :func:`p2_kernels`."""
    real, xt, suffix = {"f64": ("double", "double", "f64"), "f32": ("float", "double", "f32"),
                        "f32g": ("float", "float", "f32g")}[precision]
    head = "#define REAL %s\n" % real + (_P2_COMMON % {"S": suffix}).replace("static __inline__ ", "static inline ")
    stiff = (_P2_STIFF % {"name": "p2_km_stiff_" + suffix, "X": xt, "S": suffix}).replace(
        "\nvoid ", "\nstatic inline void ", 1)
    mass = (_P2_MASS % {"name": "p2_km_mass_" + suffix, "X": xt, "S": suffix}).replace(
        "\nvoid ", "\nstatic inline void ", 1)
    name = "p2_km_" + suffix
    entry = ("\nvoid %s(double A[1][1], double M[1][1], %s *x[2], int j, int k) {\n"
             "  p2_km_stiff_%s(A, x, j, k);\n  p2_km_mass_%s(M, x, j, k);\n}\n"
             % (name, xt, suffix, suffix))
    return head + stiff + mass + entry + "#undef REAL\n", name


class Problem(object):
    pass


def build_p1(op2, n, coords=None, elem=None, stiffness=False):
    """P1 mass Mat + RHS Dat on the n x n square."""
    if coords is None:
        coords, elem = square_p1(n)
    P = Problem()
    P.nodes = op2.Set(len(coords), 1, "nodes")
    P.vnodes = op2.Set(len(coords), 2, "vnodes")
    P.elements = op2.Set(len(elem), 1, "elements")
    P.elem_node = op2.Map(P.elements, P.nodes, 3, elem, "elem_node")
    P.elem_vnode = op2.Map(P.elements, P.vnodes, 3, elem, "elem_vnode")
    P.sparsity = op2.Sparsity((P.elem_node, P.elem_node), "p1_sparsity")
    P.mat = op2.Mat(P.sparsity, np.float64, "mass")
    P.coords = op2.Dat(P.vnodes, coords, np.float64, "coords")
    P.f = op2.Dat(P.nodes, np.sin(np.pi * coords[:, 0]) * np.sin(np.pi * coords[:, 1]), np.float64, "f")
    P.b = op2.Dat(P.nodes, np.zeros(len(coords)), np.float64, "b")
    P.k_mass = op2.Kernel(P1_MASS, "p1_mass")
    P.k_rhs = op2.Kernel(P1_RHS, "p1_rhs")
    if stiffness:
        P.stiff = op2.Mat(P.sparsity, np.float64, "stiffness")
        P.k_stiff = op2.Kernel(P1_STIFF, "p1_stiff")
    P.n_elem, P.n_nodes = len(elem), len(coords)
    return P


def assemble_p1_stiffness(op2, P):
    op2.par_loop(P.k_stiff, P.elements(3, 3),
                 P.stiff((P.elem_node[op2.i[0]], P.elem_node[op2.i[1]]), op2.INC),
                 P.coords(P.elem_vnode, op2.READ))


def assemble_p1(op2, P):
    op2.par_loop(P.k_mass, P.elements(3, 3),
                 P.mat((P.elem_node[op2.i[0]], P.elem_node[op2.i[1]]), op2.INC),
                 P.coords(P.elem_vnode, op2.READ))
    op2.par_loop(P.k_rhs, P.elements(3), P.b(P.elem_node[op2.i[0]], op2.INC),
                 P.coords(P.elem_vnode, op2.READ), P.f(P.elem_node, op2.READ))


def build_p2(op2, n, seed=0, precision="f64", coords=None, elem=None):
    """P2 stiffness + mass Mats on one Sparsity."""
    if coords is None:
        coords, elem = square_p2(n, seed)
    P = Problem()
    P.dofs = op2.Set(len(coords), 1, "dofs")
    P.vdofs = op2.Set(len(coords), 2, "vdofs")
    P.elements = op2.Set(len(elem), 1, "elements")
    P.elem_dof = op2.Map(P.elements, P.dofs, 6, elem, "elem_dof")
    P.elem_vdof = op2.Map(P.elements, P.vdofs, 6, elem, "elem_vdof")
    P.sparsity = op2.Sparsity((P.elem_dof, P.elem_dof), "p2_sparsity")
    P.K = op2.Mat(P.sparsity, np.float64, "stiffness")
    P.M = op2.Mat(P.sparsity, np.float64, "mass")
    xdt = np.float32 if precision == "f32g" else np.float64
    P.coords = op2.Dat(P.vdofs, coords.astype(xdt), xdt, "coords")
    (ks, ns), (km, nm) = p2_kernels(precision)
    P.k_stiff = op2.Kernel(ks, ns)
    P.k_mass = op2.Kernel(km, nm)
    kkm, nkm = p2_km_kernel(precision)
    P.k_km = op2.Kernel(kkm, nkm)
    P.n_elem, P.n_dofs = len(elem), len(coords)
    return P


def assemble_p2(op2, P, fused=True):
    """K and M: by one par_loop computing both (``fused``, the default), or
    by one par_loop per Mat."""
    rows = (P.elem_dof[op2.i[0]], P.elem_dof[op2.i[1]])
    if fused:
        op2.par_loop(P.k_km, P.elements(6, 6), P.K(rows, op2.INC), P.M(rows, op2.INC),
                     P.coords(P.elem_vdof, op2.READ))
        return
    for mat, k in ((P.K, P.k_stiff), (P.M, P.k_mass)):
        op2.par_loop(k, P.elements(6, 6), mat(rows, op2.INC), P.coords(P.elem_vdof, op2.READ))


def assembly_bytes(n_elem, arity, n_nodes, nnz, coord_bytes=8, nmats=1):
    """Algorithmic bytes of Mat assembly: the map, the coordinates, the CSR
    values read and written, and the CSR structure (rowptr + colidx), per
    Mat; the map and coordinates are counted once per assembly loop."""
    per_loop = n_elem * arity * 4 + n_nodes * 2 * coord_bytes
    per_mat = nnz * 8 * 2 + (n_nodes + 1) * 4 + nnz * 4
    return nmats * (per_loop + per_mat)


def km_bytes(n_elem, arity, n_nodes, nnz, coord_bytes=8, nmats=2):
    """Algorithmic bytes of assembling ``nmats`` Mats on ONE Sparsity over
    the same elements (P2 stiffness + mass): the map and the coordinates
    once, the CSR structure once, and every Mat's values read and written.
    At 1024 x 1024 P2 this is 50.3 MB + 67.2 MB + 2 x 772.0 MB + 209.8 MB =
    1.871 GB."""
    return (n_elem * arity * 4 + n_nodes * 2 * coord_bytes + nmats * nnz * 8 * 2
            + (n_nodes + 1) * 4 + nnz * 4)


def rhs_bytes(n_elem, n_nodes):
    """P1 RHS: map, coords, f read, b read-modify-write."""
    return n_elem * 3 * 4 + n_nodes * 16 + n_nodes * 8 + n_nodes * 16
