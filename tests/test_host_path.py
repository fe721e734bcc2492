"""Host-side par_loop path: the bound-loop key the cached-call fast path
looks loops up by (pyop2_b200.b200._loop_key).  Loops may share a bound
loop only when they are the same loop over the same objects; a fresh Global
per call must not defeat the cache.  CPU only: keys touch no device."""

import numpy as np
import pytest

from pyop2_b200 import backends


@pytest.fixture(scope="module")
def op2():
    from pyop2_b200 import op2 as _op2
    if backends.get_backend() == "pyop2_b200.void":
        backends.set_backend("b200")
    return _op2


def test_loop_key_identity_rules(op2):
    from pyop2_b200 import b200
    from pyop2_b200 import configuration as cfg
    cells, edges = op2.Set(8, 1, "cells"), op2.Set(10, 1, "edges")
    m = op2.Map(edges, cells, 2, np.arange(20, dtype=np.int32) % 8, "m")
    m2 = op2.Map(edges, cells, 2, np.arange(20, dtype=np.int32) % 8, "m2")
    x = op2.Dat(cells, np.zeros(8), np.float64, "x")
    y = op2.Dat(cells, np.zeros(8), np.float64, "y")
    k = op2.Kernel("void k(double *a, double *b, double *g) { }", "k")

    def key(dat, mp, acc, g, its=False):
        idx = op2.i[0] if its else 0
        args = (dat(mp[idx], acc), x(mp[1], op2.READ), g(op2.INC))
        return b200._loop_key(k, edges, (2,) if its else (), args)

    g1, g2 = op2.Global(1, 0.0, np.float64, "g"), op2.Global(1, 5.0, np.float64, "g")
    base = key(x, m, op2.INC, g1)
    assert key(x, m, op2.INC, g1) == base          # same loop, same objects
    assert key(x, m, op2.INC, g2) == base          # a fresh Global reuses the loop
    assert key(y, m, op2.INC, g1) != base          # another Dat
    assert key(x, m2, op2.INC, g1) != base         # another Map with equal values
    assert key(x, m, op2.WRITE, g1) != base        # another access mode
    assert key(x, m, op2.INC, g1, its=True) != base  # an iteration-space index
    g3 = op2.Global(1, 0, np.int32, "g")
    assert key(x, m, op2.INC, g3) != base          # a Global of another type
    old = cfg.cfg['inc_mode']
    try:
        cfg.configure(inc_mode="lma" if old != "lma" else "atomic")
        assert key(x, m, op2.INC, g1) != base      # the configuration is part of the key
    finally:
        cfg.configure(inc_mode=old)
    assert key(x, m, op2.INC, g1) == base


def test_argument_fast_paths_keep_the_reference_errors(op2):
    from pyop2_b200 import exceptions
    s, t = op2.Set(4), op2.Set(3)
    m = op2.Map(s, t, 2, np.zeros(8, np.int32), "m")
    d = op2.Dat(t, np.zeros(3), np.float64, "d")
    a = d(m[1], op2.INC)
    assert a.map is m and a.idx == 1 and a.access is op2.INC and a.data is d
    with pytest.raises(exceptions.IndexValueError):
        m[2]
    with pytest.raises(exceptions.IndexTypeError):
        m["0"]
    assert m[np.int32(1)].idx == 1
    with pytest.raises(exceptions.ModeValueError):
        d(m[0], op2.MIN)
    # a Dat on the wrong set is caught where the reference catches it: when
    # the loop checks its arguments (pyop2/base.py ParLoop.check_args)
    from pyop2_b200 import b200
    bad = op2.Dat(s, np.zeros(4), np.float64)(m[0], op2.READ)
    with pytest.raises(exceptions.MapValueError):
        b200.ParLoop(op2.Kernel("void kb(double *a) { }", "kb"), s, bad)
    g = op2.Global(1, 2, np.int32, "g")
    assert g.data.dtype == np.int32 and g.data[0] == 2 and g.data.shape == (1,)
    assert op2.Global(1, 2.5).data.dtype == np.float64
