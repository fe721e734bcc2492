"""Host-side API semantics (validation and errors of pyop2/base.py, as the
reference's test/unit/test_api.py checks them).  CPU only: the data classes
touch no device until a loop runs."""

import numpy as np
import pytest

from pyop2_b200 import backends, base, exceptions


@pytest.fixture(scope="module")
def op2():
    from pyop2_b200 import op2 as _op2
    if backends.get_backend() == "pyop2_b200.void":
        backends.set_backend("b200")
    return _op2


def test_access_modes(op2):
    for m in ("READ", "WRITE", "RW", "INC", "MIN", "MAX"):
        assert getattr(op2, m)._mode == m
    with pytest.raises(exceptions.ModeValueError):
        base.Access("ILLEGAL_ACCESS")


def test_set(op2):
    with pytest.raises(exceptions.SizeTypeError):
        op2.Set('illegalsize')
    with pytest.raises(TypeError):
        op2.Set(1, 'illegaldim')
    with pytest.raises(exceptions.NameTypeError):
        op2.Set(1, 1, 2)
    s = op2.Set(5, (2, 3), 'foo')
    assert s.dim == (2, 3) and s.cdim == 6 and s.size == 5 and s.sizes == (5, 5, 5, 5)


def test_dat(op2):
    s = op2.Set(5, 2, 'foo')
    with pytest.raises(exceptions.SetTypeError):
        op2.Dat('illegalset', 1)
    with pytest.raises(exceptions.NameTypeError):
        op2.Dat(s, None, None, 2)
    d = op2.Dat(s, np.arange(10), np.int32)
    assert d.dtype == np.int32 and d.data.shape == (5, 2)
    with pytest.raises(exceptions.DataTypeError):
        op2.Dat(s, [1] * 10, 'illegal_type')
    with pytest.raises(exceptions.DataValueError):
        op2.Dat(s, [1] * 3)
    d2 = op2.Dat(s, [1.5] * 10, np.int32)
    assert d2.dtype == np.int32
    other = op2.Set(4)
    m = op2.Map(op2.Set(3), other, 1, [0, 1, 2])
    with pytest.raises(exceptions.MapValueError):
        d(m, op2.READ)
    with pytest.raises(exceptions.ModeValueError):
        d(op2.IdentityMap, op2.MIN)
    ro = d.data_ro
    with pytest.raises((RuntimeError, ValueError)):
        ro[0] = 1


def test_map(op2):
    s, t = op2.Set(3), op2.Set(4)
    with pytest.raises(exceptions.SetTypeError):
        op2.Map('illegalset', t, 1, [])
    with pytest.raises(exceptions.DimTypeError):
        op2.Map(s, t, 'illegaldim', [])
    with pytest.raises(exceptions.DataValueError):
        op2.Map(s, t, 1, [1, 2])
    m = op2.Map(s, t, 2, [0, 1, 2, 3, 0, 1], 'm')
    assert m.values.shape == (3, 2) and m.values.dtype == np.int32
    with pytest.raises(exceptions.IndexValueError):
        m[2]
    with pytest.raises(exceptions.IndexValueError):
        m[op2.i[2]]
    with pytest.raises(exceptions.MapValueError):
        op2.Map(s, t, 1)  # the device backend needs values
    m2 = op2.Map(s, t, 2, [0, 1, 2, 3, 0, 1], 'm')
    assert m == m2
    assert m != op2.Map(s, t, 2, [0, 1, 2, 3, 0, 1], 'other')


def test_global_and_const(op2):
    g = op2.Global(2, [1, 2], np.int32, 'g')
    assert (g.data == [1, 2]).all()
    with pytest.raises(exceptions.DataValueError):
        op2.Global(2, [1, 2, 3])
    with pytest.raises(exceptions.ModeValueError):
        g(op2.RW)
    c = op2.Const(2, [1, 2], 'c_api_test', np.int32)
    with pytest.raises(op2.Const.NonUniqueNameError):
        op2.Const(1, 1, 'c_api_test')
    c.remove_from_namespace()
    c2 = op2.Const(1, 3, 'c_api_test')
    c2.remove_from_namespace()


def test_sparsity_and_mat_validation(op2):
    s = op2.Set(3)
    with pytest.raises(TypeError):
        op2.Sparsity(('illegalrmap', 'illegalcmap'))
    with pytest.raises(exceptions.SparsityTypeError):
        op2.Mat('illegalsparsity')


def test_parloop_checks_itersets(op2):
    a, b, c = op2.Set(3), op2.Set(4), op2.Set(3)
    m = op2.Map(a, b, 1, [0, 1, 2])
    d = op2.Dat(b, np.zeros(4))
    k = op2.Kernel("void k(double *x) {}", "k")
    from pyop2_b200 import b200
    with pytest.raises(exceptions.MapValueError):
        b200.ParLoop(k, c, d(m[0], op2.READ))


def test_kernel_cache(op2):
    k1 = op2.Kernel("void k(double *x) {}", "k")
    k2 = op2.Kernel("void k(double *x) {}", "k")
    assert k1 is k2
