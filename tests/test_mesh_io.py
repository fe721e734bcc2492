"""Mesh and data ingestion: the ``fromhdf5`` constructors (the cases of the
reference's test/unit/test_hdf5.py) and the Triangle reader
(pyop2/demo/triangle_reader.py).  h5py is not installed here, so the HDF5
cases run on an in-memory object with h5py's File interface (datasets with
``shape``, ``attrs`` and ``[()]``); with h5py present the same cases also
run on a real file.  CPU only: the data classes touch no device."""

import numpy as np
import pytest

from pyop2_b200 import backends, exceptions
from pyop2_b200 import triangle_reader as tr
from pyop2_b200.workloads import airfoil, meshes


@pytest.fixture(scope="module")
def op2():
    from pyop2_b200 import op2 as _op2
    if backends.get_backend() == "pyop2_b200.void":
        backends.set_backend("b200")
    return _op2


class H5Dataset(object):
    def __init__(self, data, attrs=None):
        self._data = np.asarray(data)
        self.shape = self._data.shape
        self.attrs = dict(attrs or {})

    def __getitem__(self, key):
        return self._data[key]


class H5File(dict):
    @classmethod
    def from_layout(cls, layout):
        return cls({k: H5Dataset(a, attrs) for k, (a, attrs) in layout.items()})


def _reference_file():
    """The datasets of test_hdf5.py's fixture (test/unit/test_hdf5.py:52-64)."""
    return H5File({
        "dat": H5Dataset(np.arange(10, dtype=np.float64).reshape(5, 2), {"type": "double"}),
        "soadat": H5Dataset(np.arange(10, dtype=np.float64).reshape(5, 2), {"type": "double:soa"}),
        "set": H5Dataset(np.array((5,)), {"dim": 2}),
        "myconstant": H5Dataset(np.arange(3)),
        "map": H5Dataset(np.array((1, 2, 2, 3)).reshape(2, 2)),
    })


def _check_reference_cases(op2, f):
    s = op2.Set.fromhdf5(f, name="set")
    assert s.size == 5 and s.dim == (2,)
    st = op2.Set(5, 2, "foo")
    d = op2.Dat.fromhdf5(st, f, "dat")
    assert d.dtype == np.float64 and not d.soa
    assert d.data.shape == (5, 2) and d.data.sum() == 9 * 10 / 2
    d = op2.Dat.fromhdf5(st, f, "soadat")
    assert d.soa and d.data.shape == (5, 2) and d.data.sum() == 9 * 10 / 2
    c = op2.Const.fromhdf5(f, "myconstant")
    try:
        assert c.data.sum() == 3 and c.dim == (3,)
    finally:
        c.remove_from_namespace()
    iterset, dataset = op2.Set(2, 1, "iterset"), op2.Set(3, 1, "dataset")
    m = op2.Map.fromhdf5(iterset, dataset, f, name="map")
    assert m.iterset == iterset and m.dataset == dataset and m.dim == 2
    assert m.values.sum() == sum((1, 2, 2, 3)) and m.name == "map"


def test_fromhdf5_reference_cases(op2):
    _check_reference_cases(op2, _reference_file())


def test_fromhdf5_errors(op2):
    f = H5File({"bad_set": H5Dataset(np.array((5, 6))), "flat_map": H5Dataset(np.arange(4)),
                "scalar": H5Dataset(np.float64(1.0))})
    with pytest.raises(exceptions.SizeTypeError):
        op2.Set.fromhdf5(f, "bad_set")
    with pytest.raises(exceptions.DimTypeError):
        op2.Map.fromhdf5(op2.Set(4), op2.Set(4), f, "flat_map")
    with pytest.raises(exceptions.DimTypeError):
        op2.Const.fromhdf5(f, "scalar")


def test_fromhdf5_real_file(op2, tmp_path):
    h5py = pytest.importorskip("h5py")
    path = str(tmp_path / "tmp_hdf5.h5")
    with h5py.File(path, "w") as f:
        for name, ds in _reference_file().items():
            f.create_dataset(name, data=ds[()])
            for k, v in ds.attrs.items():
                f[name].attrs[k] = v
    with h5py.File(path, "r") as f:
        _check_reference_cases(op2, f)


def test_airfoil_mesh_file_layout(op2):
    """The airfoil problem declared as pyop2/demo/airfoil.py:45-75 declares
    it from a mesh file equals the one declared directly from the grid."""
    from pyop2_b200 import base
    for c in list(base.Const._defs):
        c.remove_from_namespace()
    g = meshes.airfoil_grid(12, 6, 3)
    A = airfoil.build_from_hdf5(op2, H5File.from_layout(airfoil.hdf5_layout(g, seed=3)))
    try:
        assert (A.nodes.size, A.nodes.dim) == (g.nnodes, (2,))
        assert (A.edges.size, A.bedges.size, A.cells.size) == (g.nedges, g.nbedges, g.ncells)
        assert A.vcells.dim == (4,)
        for name, arity, src in (("pedge", 2, g.pedge), ("pecell", 2, g.pecell), ("pevcell", 2, g.pecell),
                                 ("pbedge", 2, g.pbedge), ("pbecell", 1, g.pbecell), ("pcell", 4, g.pcell)):
            m = getattr(A, name)
            assert m.dim == arity
            np.testing.assert_array_equal(m.values.ravel(), np.asarray(src).ravel())
        assert A.pevcell.dataset is A.vcells and A.pcell.dataset is A.vnodes
        np.testing.assert_array_equal(A.p_x.data.ravel(), np.asarray(g.x).ravel())
        np.testing.assert_array_equal(A.p_q.data, airfoil.initial_q(g.ncells, 3))
        assert A.p_bound.dtype == np.int32 and not A.p_q.soa
        assert [c.name for c in A.consts] == ["gam", "gm1", "cfl", "eps", "mach", "alpha", "qinf"]
        assert A.consts[-1].dim == (4,) and A.consts[0].data[0] == airfoil.GAM
    finally:
        for c in A.consts:
            c.remove_from_namespace()


def test_triangle_round_trip_and_objects(op2, tmp_path):
    coords, elem = meshes.square_p1(7)
    prefix = str(tmp_path / "sq")
    tr.write_triangle(prefix, coords, elem)
    c2, e2 = tr.read_triangle_arrays(prefix)
    np.testing.assert_array_equal(c2, coords)
    np.testing.assert_array_equal(e2, elem)
    nodes, vnodes, x, elements, en, evn = tr.read_triangle(prefix, op2)
    assert (nodes.size, vnodes.dim, elements.size) == (len(coords), (2,), len(elem))
    assert en.dim == evn.dim == 3 and en.dataset is nodes and evn.dataset is vnodes
    np.testing.assert_array_equal(x.data, coords)
    np.testing.assert_array_equal(en.values, elem)


def test_triangle_comments_attributes_and_order(tmp_path):
    """Comment lines, boundary markers, element attributes (as gmsh2triangle
    writes them) and records out of numbering order."""
    prefix = str(tmp_path / "g")
    with open(prefix + ".node", "w") as h:
        h.write("# vertices\n4 2 0 1\n")
        h.write("3 1.0 1.0 1\n1 0.0 0.0 1\n\n# comment inside\n2 1.0 0.0 1\n4 0.0 1.0 1\n")
    with open(prefix + ".ele", "w") as h:
        h.write("2 3 1\n2 1 3 4 7\n1 1 2 3 7\n# end\n")
    coords, elem = tr.read_triangle_arrays(prefix)
    np.testing.assert_array_equal(coords, [[0, 0], [1, 0], [1, 1], [0, 1]])
    np.testing.assert_array_equal(elem, [[0, 1, 2], [0, 2, 3]])
