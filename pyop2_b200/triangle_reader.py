"""Triangle (.node / .ele) mesh files into op2 data structures.

Restates the reader of the reference's demos (pyop2/demo/triangle_reader.py:
39-85): the ``.node`` file gives the vertex coordinates (1-based vertex
numbers, attributes and boundary markers ignored), the ``.ele`` file the
triangles (1-based triangle and vertex numbers); ``#`` starts a comment
line.  The files are parsed with numpy instead of line by line, so meshes of
millions of triangles load in seconds.
"""

import numpy as np


def _rows(path):
    """Header fields and the data rows (comment and blank lines dropped) of
    a Triangle file."""
    with open(path) as h:
        lines = [ln for ln in h.read().splitlines() if ln.strip() and not ln.lstrip().startswith('#')]
    header = [int(v) for v in lines[0].split()]
    body = " ".join(lines[1:])
    return header, body


def read_triangle_arrays(f):
    """(coords [n, 2] float64, elem_node [m, 3] int32, 0-based) of the mesh
    with file prefix ``f``."""
    (num_nodes, *_), body = _rows(f + '.node')
    vals = np.array(body.split(), dtype=np.float64)
    per = vals.size // num_nodes if num_nodes else 3
    vals = vals.reshape(num_nodes, per)
    coords = np.zeros((num_nodes, 2))
    coords[vals[:, 0].astype(np.int64) - 1] = vals[:, 1:3]
    (num_tri, nodes_per_tri, *_), body = _rows(f + '.ele')
    # integers, possibly written with a decimal point (attributes)
    vals = np.array(body.split(), dtype=np.float64).astype(np.int64)
    per = vals.size // num_tri if num_tri else 1 + nodes_per_tri
    vals = vals.reshape(num_tri, per)
    elem = np.zeros((num_tri, 3), dtype=np.int32)
    elem[vals[:, 0] - 1] = vals[:, 1:4] - 1
    return coords, elem


def read_triangle(f, op2=None):
    """Read the Triangle files with prefix ``f`` into op2 objects, returned
    as the reference's reader returns them:
    ``(nodes, vnodes, coords, elements, elem_node, elem_vnode)`` with types
    ``(Set, Set, Dat, Set, Map, Map)``."""
    if op2 is None:
        from . import op2
    coords, elem = read_triangle_arrays(f)
    num_nodes, num_tri = coords.shape[0], elem.shape[0]
    nodes = op2.Set(num_nodes, 1, "nodes")
    vnodes = op2.Set(num_nodes, 2, "vnodes")
    dcoords = op2.Dat(vnodes, coords, np.float64, "coords")
    elements = op2.Set(num_tri, 1, "elements")
    elem_node = op2.Map(elements, nodes, 3, elem, "elem_node")
    elem_vnode = op2.Map(elements, vnodes, 3, elem, "elem_vnode")
    return nodes, vnodes, dcoords, elements, elem_node, elem_vnode


def write_triangle(f, coords, elem):
    """Write ``coords`` [n, 2] and 0-based ``elem`` [m, 3] as Triangle files
    with prefix ``f`` (1-based numbers, no attributes or markers)."""
    coords = np.asarray(coords, dtype=np.float64)
    elem = np.asarray(elem, dtype=np.int64)
    with open(f + '.node', 'w') as h:
        h.write("%d 2 0 0\n" % coords.shape[0])
        np.savetxt(h, np.column_stack([np.arange(1, coords.shape[0] + 1), coords]),
                   fmt=["%d", "%.17g", "%.17g"])
    with open(f + '.ele', 'w') as h:
        h.write("%d 3 0\n" % elem.shape[0])
        np.savetxt(h, np.column_stack([np.arange(1, elem.shape[0] + 1), elem + 1]), fmt="%d")
