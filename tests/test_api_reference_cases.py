"""The op2 API's construction, validation and error behaviour case by case
as the reference's unit tests check it (test/unit/test_api.py: Init, Access,
Set, Dat, Sparsity, Mat, Const, Global, Map, IterationSpace, Kernel,
illegal iteration-set Maps, Solver).  The MPI communicator cases are not
restated: this backend runs one process per GPU without mpi4py, and
``op2.MPI`` reports a serial run.  CPU only: nothing here touches a device
(a Sparsity builds its CSR on the device at first use, not at
construction)."""

import subprocess
import sys

import numpy as np
import pytest

from pyop2_b200 import backends, base, exceptions


@pytest.fixture(scope="module")
def op2():
    from pyop2_b200 import op2 as _op2
    if backends.get_backend() == "pyop2_b200.void":
        backends.set_backend("b200")
    return _op2


@pytest.fixture(params=[1, 2, (2, 3)])
def aset(op2, request):
    return op2.Set(5, request.param, "foo")


@pytest.fixture
def iterset(op2):
    return op2.Set(2, 1, "iterset")


@pytest.fixture
def dataset(op2):
    return op2.Set(3, 1, "dataset")


@pytest.fixture
def m(op2, iterset, dataset):
    return op2.Map(iterset, dataset, 2, [1] * 2 * iterset.size, "m")


@pytest.fixture
def sparsity(op2, m):
    return op2.Sparsity((m, m))


def _cdim(s):
    return int(np.prod(s.dim))


# ------------------------------------------------------------------ init
def test_use_before_init_and_invalid_backend():
    """Before init, creating a Set raises RuntimeError; init with an unknown
    backend raises ImportError (a fresh interpreter: the other tests select
    the backend for the whole process)."""
    code = ("import pytest\n"
            "from pyop2_b200 import op2\n"
            "with pytest.raises(RuntimeError):\n"
            "    op2.Set(1)\n"
            "with pytest.raises(ImportError):\n"
            "    op2.init(backend='invalid_backend')\n")
    subprocess.check_call([sys.executable, "-c", code])


def test_serial_run(op2):
    assert not op2.MPI.parallel


# ---------------------------------------------------------------- access
@pytest.mark.parametrize("mode", ["READ", "WRITE", "RW", "INC", "MIN", "MAX"])
def test_access_repr(op2, mode):
    assert repr(base.Access(mode)) == "Access('%s')" % mode


# ------------------------------------------------------------------- Set
def test_set_arguments(op2):
    with pytest.raises(exceptions.SizeTypeError):
        op2.Set("illegalsize")
    with pytest.raises(TypeError):
        op2.Set(1, "illegaldim")
    with pytest.raises(TypeError):
        op2.Set(1, (1, "illegaldim"))
    with pytest.raises(exceptions.NameTypeError):
        op2.Set(1, 1, 2)
    assert op2.Set(1, 1).dim == (1,)
    assert op2.Set(1, [2, 3]).dim == (2, 3)


def test_set_repr_str_and_identity(op2, aset):
    assert repr(aset) and str(aset)
    copy = op2.Set(aset.size, aset.dim, aset.name)
    assert aset == aset and aset != copy


# ------------------------------------------------------------------- Dat
def test_dat_arguments(op2, aset):
    with pytest.raises(exceptions.SetTypeError):
        op2.Dat("illegalset", 1)
    with pytest.raises(exceptions.NameTypeError):
        op2.Dat(aset, name=2)
    with pytest.raises(exceptions.DataTypeError):
        op2.Dat(aset, dtype="illegal_type")
    with pytest.raises(exceptions.DataValueError):
        op2.Dat(aset, [1] * (aset.size * _cdim(aset) + 1))


def test_dat_default_data_and_types(op2, aset):
    n = aset.size * _cdim(aset)
    d = op2.Dat(aset)
    assert d.data.size == n and d.data.dtype == np.float64 and d.dtype == np.double
    assert op2.Dat(aset, dtype=np.int32).data.dtype == np.int32
    assert op2.Dat(aset, [1.0] * n).dtype == np.double
    assert op2.Dat(aset, [1] * n).dtype == np.asarray([1]).dtype
    assert op2.Dat(aset, [1] * n, np.double).dtype == np.float64
    assert op2.Dat(aset, [1.5] * n, np.int32).dtype == np.int32
    assert op2.Dat(aset, [1.0] * n).data.shape == (aset.size,) + aset.dim


def test_dat_properties(op2, aset):
    n = aset.size * _cdim(aset)
    d = op2.Dat(aset, [1] * n, "double", "bar")
    assert d.dataset == aset and d.dtype == np.float64 and d.name == "bar" and d.data.sum() == n


def test_dat_map_from_another_set(op2, aset):
    d = op2.Dat(aset)
    to_other = op2.Map(op2.Set(3), op2.Set(2), 1, [0, 0, 0])
    with pytest.raises(exceptions.MapValueError):
        d(to_other, op2.READ)


def test_dat_read_only_then_writable(op2, aset):
    d = op2.Dat(aset, np.arange(_cdim(aset) * aset.size), dtype=np.int32)
    x = d.data_ro
    with pytest.raises((RuntimeError, ValueError)):
        x[0] = 1
    x = d.data
    x[0] = -100
    assert (d.data_ro[0] == -100).all()


def test_dat_arithmetic_shape_mismatch(op2):
    """test/unit/test_linalg.py:86-100, 175-189: operands of the same size
    but different shapes, (1, 2) and (2, 1) per element, raise ValueError
    (the values broadcast to (2, 2) per element, which fits neither Dat).
    Such operands take the host path, so this runs without a device."""
    import operator
    n = 8
    for op in (operator.add, operator.sub, operator.mul, operator.truediv,
               operator.iadd, operator.isub, operator.imul, operator.itruediv):
        x2 = op2.Dat(op2.Set(n, (1, 2)), np.arange(2 * n) + 1.0, np.float64, "x")
        y2 = op2.Dat(op2.Set(n, (2, 1)), np.arange(2 * n) + 1.0, np.float64, "y")
        with pytest.raises(ValueError):
            op(x2, y2)


@pytest.mark.parametrize("name", ["add", "sub", "mul", "truediv"])
def test_dat_arithmetic_mixed_types(op2, name):
    """test/unit/test_linalg.py:118-148, 205-243: the result keeps the left
    operand's type (the right one is cast to it first), in place too; an
    integer Dat divides by floor division, as ``/`` between integer arrays
    did under the reference's Python 2.  Mixed-type operands take the host
    path, so this runs without a device."""
    import operator
    s = op2.Set(8)

    def pair():
        return (op2.Dat(s, np.arange(1, 9), np.float64, "y"),
                op2.Dat(s, [-4, -3, -2, -1, 1, 2, 3, 4], np.int64, "yi"))
    op, iop = getattr(operator, name), getattr(operator, "i" + name)
    y, yi = pair()
    assert op(y, yi).data.dtype == np.float64
    assert op(yi, y).data.dtype == np.int64
    y, yi = pair()
    assert iop(y, yi).data.dtype == np.float64
    y, yi = pair()
    r = iop(yi, y)
    assert r is yi and yi.data.dtype == np.int64
    a, b = np.array([-4, -3, -2, -1, 1, 2, 3, 4]), np.arange(1, 9)
    want = {"add": a + b, "sub": a - b, "mul": a * b, "truediv": a // b}[name]
    np.testing.assert_array_equal(yi.data.ravel(), want)
    y, yi = pair()
    np.testing.assert_array_equal(op(yi, y).data.ravel(), want)


# -------------------------------------------------------------- Sparsity
def test_sparsity_map_arguments(op2, m):
    with pytest.raises(TypeError):
        op2.Sparsity(("illegalrmap", m))
    with pytest.raises(TypeError):
        op2.Sparsity((m, "illegalcmap"))


def test_sparsity_forms(op2, m, iterset):
    s = op2.Sparsity(m, "foo")
    assert s.maps[0] == (m, m) and s.dims == (1, 1) and s.name == "foo"
    s = op2.Sparsity((m, m), "foo")
    assert s.maps[0] == (m, m) and s.dims == (1, 1) and s.name == "foo"
    md = op2.Map(iterset, op2.Set(1, 1, "dataset2"), 1, [1] * iterset.size, "md")
    s = op2.Sparsity((m, md), "foo")
    assert s.maps[0] == (m, md) and s.dims == (1, 1)
    s = op2.Sparsity(((m, m), (m, m)), "foo")
    assert s.maps == [(m, m), (m, m)] and s.dims == (1, 1)
    mi = op2.Map(op2.Set(3, 1, "iterset2"), m.dataset, 1, [1] * 3, "mi")
    s = op2.Sparsity(((m, m), (mi, mi)), "foo")
    assert len(s.maps) == 2 and s.dims == (1, 1)


def test_sparsity_inconsistent_maps(op2, m, iterset):
    mi = op2.Map(op2.Set(3, 1, "iterset2"), m.dataset, 1, [1] * 3, "mi")
    md = op2.Map(iterset, op2.Set(1, 1, "dataset2"), 1, [1] * iterset.size, "md")
    with pytest.raises(RuntimeError):
        op2.Sparsity((m, mi))                 # one iteration set per pair
    with pytest.raises(RuntimeError):
        op2.Sparsity(((m, m), (md, m)))       # one row data set
    with pytest.raises(RuntimeError):
        op2.Sparsity(((m, m), (m, md)))       # one column data set


# ------------------------------------------------------------------- Mat
def test_mat_arguments_and_properties(op2, sparsity):
    with pytest.raises(TypeError):
        op2.Mat("illegalsparsity")
    with pytest.raises(exceptions.NameTypeError):
        op2.Mat(sparsity, name=2)
    assert op2.Mat(sparsity).dtype == np.double
    mat = op2.Mat(sparsity, "double", "bar")
    assert mat.sparsity == sparsity and mat.dtype == np.float64 and mat.name == "bar"
    wrong = op2.Map(op2.Set(2), op2.Set(3), 2, [0, 0, 0, 0])
    with pytest.raises(exceptions.MapValueError):
        mat((wrong[0], wrong[1]), op2.INC)


# ----------------------------------------------------------------- Const
def test_const_arguments(op2):
    with pytest.raises(TypeError):
        op2.Const("illegaldim", 1, "test_const_illegal_dim")
    with pytest.raises(TypeError):
        op2.Const((1, "illegaldim"), 1, "test_const_illegal_dim_tuple")
    with pytest.raises(exceptions.NameTypeError):
        op2.Const(1, 1, 2)
    with pytest.raises(exceptions.DataValueError):
        op2.Const(1, "illegal_type", "test_const_illegal_dtype", "double")
    for dim in (1, (2, 2)):
        with pytest.raises(exceptions.DataValueError):
            op2.Const(dim, [1] * (int(np.prod(dim)) + 1), "test_const_illegal_length_%d" % np.prod(dim))


def test_const_names_are_unique_until_removed(op2):
    c = op2.Const(1, 1, "test_const_nonunique_name")
    try:
        with pytest.raises(op2.Const.NonUniqueNameError):
            op2.Const(1, 1, "test_const_nonunique_name")
    finally:
        c.remove_from_namespace()
    c = op2.Const(1, 1, "test_const_remove_from_namespace")
    c.remove_from_namespace()
    c = op2.Const(1, 1, "test_const_remove_from_namespace")
    c.remove_from_namespace()
    assert c.name == "test_const_remove_from_namespace"


def _const(op2, *a):
    c = op2.Const(*a)
    c.remove_from_namespace()
    return c


def test_const_shapes_and_types(op2):
    assert _const(op2, 1, 1, "test_const_dim").dim == (1,)
    assert _const(op2, [2, 3], [1] * 6, "test_const_dim_list").dim == (2, 3)
    assert _const(op2, 1, 1.0, "test_const_float").dtype == np.double
    assert _const(op2, 1, 1, "test_const_int").dtype == np.asarray([1]).dtype
    assert _const(op2, 1, 1, "test_const_convert_int_float", "double").dtype == np.float64
    assert _const(op2, 1, 1.5, "test_const_convert_float_int", "int").dtype == np.dtype("int")
    c = _const(op2, (2, 2), [1.0] * 4, "test_const_reshape")
    assert c.dim == (2, 2) and c.data.shape == (2, 2)
    c = _const(op2, (2, 2), [1] * 4, "baz", "double")
    assert c.dim == (2, 2) and c.dtype == np.float64 and c.name == "baz" and c.data.sum() == 4


def test_const_setter(op2):
    c = _const(op2, 1, 1, "c")
    c.data = 2
    assert c.data.sum() == 2
    with pytest.raises(exceptions.DataValueError):
        c.data = [1, 2]


# ---------------------------------------------------------------- Global
def test_global_arguments(op2):
    with pytest.raises(TypeError):
        op2.Global("illegaldim")
    with pytest.raises(TypeError):
        op2.Global((1, "illegaldim"))
    with pytest.raises(exceptions.NameTypeError):
        op2.Global(1, 1, name=2)
    with pytest.raises(exceptions.DataValueError):
        op2.Global(1, "illegal_type", "double")
    for dim in (1, (2, 2)):
        with pytest.raises(exceptions.DataValueError):
            op2.Global(dim, [1] * (int(np.prod(dim)) + 1))


def test_global_shapes_and_types(op2):
    assert op2.Global(1, 1).dim == (1,)
    assert op2.Global([2, 3], [1] * 6).dim == (2, 3)
    assert op2.Global(1, 1.0).dtype == np.double
    assert op2.Global(1, 1).dtype == np.asarray([1]).dtype
    assert op2.Global(1, 1, "double").dtype == np.float64
    assert op2.Global(1, 1.5, "int").dtype == np.dtype("int")
    g = op2.Global((2, 2), [1.0] * 4)
    assert g.dim == (2, 2) and g.data.shape == (2, 2)
    g = op2.Global((2, 2), [1] * 4, "double", "bar")
    assert g.dim == (2, 2) and g.dtype == np.float64 and g.name == "bar" and g.data.sum() == 4


def test_global_setter(op2):
    g = op2.Global(1, 1)
    g.data = 2
    assert g.data.sum() == 2
    with pytest.raises(exceptions.DataValueError):
        g.data = [1, 2]


# ------------------------------------------------------------------- Map
def test_map_arguments(op2, aset, iterset, dataset):
    with pytest.raises(exceptions.SetTypeError):
        op2.Map("illegalset", aset, 1, [])
    with pytest.raises(exceptions.SetTypeError):
        op2.Map(aset, "illegalset", 1, [])
    with pytest.raises(exceptions.DimTypeError):
        op2.Map(aset, aset, "illegaldim", [])
    with pytest.raises(exceptions.DimTypeError):
        op2.Map(aset, aset, (2, 2), [])
    with pytest.raises(exceptions.NameTypeError):
        op2.Map(aset, aset, 1, [], name=2)
    with pytest.raises(exceptions.DataValueError):
        op2.Map(aset, aset, 1, "abcdefg")
    with pytest.raises(exceptions.DataValueError):
        op2.Map(iterset, dataset, 1, [1] * (iterset.size + 1))


def test_map_values_and_properties(op2, iterset, dataset):
    mf = op2.Map(iterset, dataset, 1, [1.5] * iterset.size)
    assert mf.values.dtype == np.int32 and mf.values.sum() == iterset.size
    m2 = op2.Map(iterset, dataset, 2, [1] * 2 * iterset.size, "bar")
    assert m2.dim == 2 and m2.values.shape == (iterset.size, 2)
    assert m2.iterset == iterset and m2.dataset == dataset and m2.values.sum() == 2 * iterset.size
    assert m2.name == "bar"
    assert m2[0].idx == 0
    with pytest.raises(NotImplementedError):
        m2[:]


def test_map_equality(op2, m):
    assert m == op2.Map(m.iterset, m.dataset, m.dim, m.values, m.name)
    itercopy = op2.Set(m.iterset.size, m.iterset.dim, m.iterset.name)
    assert m != op2.Map(itercopy, m.dataset, m.dim, m.values, m.name)
    assert m != op2.Map(m.iterset, m.dataset, m.dim * 2, list(m.values) * 2, m.name)
    assert m != op2.Map(m.iterset, m.dataset, m.dim, m.values, "n")


# -------------------------------------------------------- IterationSpace
def test_iteration_space(op2, aset):
    with pytest.raises(exceptions.SetTypeError):
        op2.IterationSpace("illegalset", 1)
    with pytest.raises(TypeError):
        op2.IterationSpace(aset, "illegalextents")
    with pytest.raises(TypeError):
        op2.IterationSpace(aset, (1, "illegalextents"))
    assert op2.IterationSpace(aset, 1).extents == (1,)
    assert op2.IterationSpace(aset, [2, 3]).extents == (2, 3)
    it = op2.IterationSpace(aset, (2, 3))
    assert it.iterset == aset and it.extents == (2, 3)


# ---------------------------------------------------------------- Kernel
def test_kernel(op2):
    with pytest.raises(exceptions.NameTypeError):
        op2.Kernel("", name=2)
    assert op2.Kernel("", "foo").name == "foo"


# ------------------------------------------- illegal iteration-set Maps
def test_loop_args_on_the_wrong_iteration_set(op2, sparsity):
    from pyop2_b200 import b200
    s1, s2 = op2.Set(2), op2.Set(3)
    dat = op2.Dat(s1)
    mp = op2.Map(s2, s1, 1, [0, 0, 0])
    k = op2.Kernel("void k() { }", "k")
    with pytest.raises(exceptions.MapValueError):
        b200.ParLoop(k, s1, dat(mp, op2.READ))
    mat = op2.Mat(sparsity)
    rmap, cmap = sparsity.maps[0]
    with pytest.raises(exceptions.MapValueError):
        b200.ParLoop(k, s1(3, 3), mat((rmap[op2.i[0]], cmap[op2.i[1]]), op2.INC))


# ---------------------------------------------------------------- Solver
def test_solver_parameters(op2):
    assert op2.Solver().parameters == base.DEFAULT_SOLVER_PARAMETERS
    params = {"linear_solver": "gmres", "maximum_iterations": 25}
    for s in (op2.Solver(params), op2.Solver(linear_solver="gmres", maximum_iterations=25)):
        assert s.parameters["linear_solver"] == "gmres" and s.parameters["maximum_iterations"] == 25
    s = op2.Solver()
    s.update_parameters(params)
    assert s.parameters["linear_solver"] == "gmres" and s.parameters["maximum_iterations"] == 25
    with pytest.raises(RuntimeError):
        op2.Solver(params, linear_solver="cgs")


# ------------------------------------------------- Kernel / Sparsity caches
def test_kernel_cache(op2):
    """test/unit/test_caching.py:542-580: a Kernel is cached by its code and
    name together."""
    cache = base.Kernel._cache
    cache.clear()
    code = "void k(void *x) {}"
    assert op2.Kernel(code, "k") is op2.Kernel(code, "k") and len(cache) == 1
    cache.clear()
    assert op2.Kernel(code, "k") is not op2.Kernel(code, "l") and len(cache) == 2
    cache.clear()
    assert op2.Kernel("void k(void *x) {}", "k") is not op2.Kernel("void l(void *x) {}", "k")
    assert len(cache) == 2
    cache.clear()
    assert op2.Kernel("void k(void *x) {}", "k") is not op2.Kernel("void l(void *x) {}", "l")
    assert len(cache) == 2


def test_sparsity_cache(op2):
    """test/unit/test_caching.py:582-651: Sparsities of the same Maps (in
    any order of the pairs) are one object; other Maps give another; Mats on
    one Sparsity share its pattern."""
    s1, s2 = op2.Set(5), op2.Set(5)
    m1 = op2.Map(s1, s2, 1, [0, 1, 2, 3, 4])
    m2 = op2.Map(s1, s2, 1, [1, 2, 3, 4, 0])
    assert op2.Sparsity(m1) is not op2.Sparsity(m2)
    assert op2.Sparsity((m1, m2)) is not op2.Sparsity((m2, m1))
    assert op2.Sparsity(((m1, m1), (m2, m2))) is not op2.Sparsity(((m2, m2), (m2, m2)))
    assert op2.Sparsity(m1) is op2.Sparsity(m1)
    assert op2.Sparsity((m1, m1)) is op2.Sparsity((m1, m1))
    assert op2.Sparsity(((m1, m1), (m2, m2))) is op2.Sparsity(((m1, m1), (m2, m2)))
    assert op2.Sparsity(((m1, m1), (m2, m2))) is op2.Sparsity(((m2, m2), (m1, m1)))
    sp = op2.Sparsity((m1, m1))
    assert op2.Mat(sp, "float64").sparsity is op2.Mat(sp, "float64").sparsity
