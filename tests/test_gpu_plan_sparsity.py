"""GPU plan and GPU Sparsity against the CPU oracle (plan.pyx and
build_sparsity_pattern_seq restated) and the reference's own compiled
sparsity_utils.cxx.

Bit-exact: partition (nelems, offset), staging (ind_map, loc_map, ind_sizes,
ind_offs, nindirect, nshared), thread colouring (thrcol, nthrcol: the same
greedy algorithm), CSR rowptr/colidx/nnz.  Block colouring is a different
(parallel) algorithm: it is checked for validity, the property the reference
tests check (test_coloring.py:84-114)."""

import numpy as np
import pytest

from conftest import py2_shuffle, reference_seed
from oracle import plan as oplan
from oracle import seq

pytestmark = pytest.mark.gpu


@pytest.fixture
def op2(backend):
    from pyop2_b200 import op2 as _op2
    return _op2


def _twin(op2, nsrc, ntgt, arity, values, name):
    """The same Map in the B200 API and in the oracle."""
    a, b = op2.Set(nsrc), op2.Set(ntgt)
    m = op2.Map(a, b, arity, values, name)
    oa, ob = seq.Set(nsrc), seq.Set(ntgt)
    return a, b, m, oa, ob, seq.Map(oa, ob, arity, values, name)


def _check_block_coloring(plan, vals_per_block):
    """No two blocks of one colour touch the same target (per race group)."""
    for c in range(plan.ncolors):
        blocks = np.where(plan.blkcol == c)[0]
        seen = {}
        for b in blocks:
            for g, t in enumerate(vals_per_block(b)):
                s = seen.setdefault(g, set())
                tt = set(np.unique(t).tolist())
                assert not (s & tt), "blocks of colour %d share a target" % c
                s |= tt


def _check_thread_coloring(plan, part, rows_of):
    for b in range(plan.nblocks):
        st = b * part
        en = st + plan.nelems[b]
        for c in range(plan.nthrcol[b]):
            sel = [e for e in range(st, en) if plan.thrcol[e] == c]
            owner = {}
            for e in sel:
                for t in set(rows_of(e)):
                    assert t not in owner, "elements %d and %d of colour %d share %d" % (owner[t], e, c, t)
                    owner[t] = e


@pytest.mark.parametrize("part", [32, 128, 256])
def test_plan_matches_oracle_indirect_inc(op2, part):
    """test_plan.py test_rhs-style args: INC through three map indices plus
    READ args, 4096 random elements."""
    from pyop2_b200 import b200
    rng = np.random.default_rng(11)
    n, nn = 4096, 1500
    vals = rng.integers(0, nn, size=(n, 3)).astype(np.int32)
    a, b, m, oa, ob, om = _twin(op2, n, nn, 3, vals, "m")
    d = op2.Dat(b, np.zeros(nn), np.float64, "d")
    c = op2.Dat(op2.Set(nn, 2), np.zeros(2 * nn), np.float64, "c")
    mc = op2.Map(a, c.dataset, 3, vals, "mc")
    od = seq.Dat(ob, np.zeros(nn))
    oc = seq.Dat(seq.Set(nn, 2), np.zeros(2 * nn))
    omc = seq.Map(oa, oc.dataset, 3, vals, "mc")
    args = [d(m[0], op2.INC), d(m[1], op2.INC), d(m[2], op2.INC),
            c(mc[0], op2.READ), c(mc[1], op2.READ), c(mc[2], op2.READ)]
    oargs = [od(om[0], seq.INC), od(om[1], seq.INC), od(om[2], seq.INC),
             oc(omc[0], seq.READ), oc(omc[1], seq.READ), oc(omc[2], seq.READ)]
    gp = b200.Plan(None, a, *args, partition_size=part)
    ref = oplan.plan(oa, oargs, partition_size=part)
    assert gp.nblocks == ref.nblocks
    for name in ("nelems", "offset", "ind_map", "loc_map", "ind_sizes", "ind_offs", "nindirect",
                 "thrcol", "nthrcol"):
        np.testing.assert_array_equal(getattr(gp, name), getattr(ref, name), err_msg=name)
    assert gp.nshared == ref.nshared
    assert gp.ncolblk.sum() == gp.nblocks
    _check_block_coloring(gp, lambda blk: [vals[blk * part:(blk + 1) * part]])
    _check_thread_coloring(gp, part, lambda e: vals[e])


def test_plan_shuffled_map_one_color(op2):
    """test_plan.py:73-83: a permutation map has no conflicts."""
    from pyop2_b200 import b200
    u = np.arange(4096, dtype=np.uint32)
    py2_shuffle(u, reference_seed)
    a, b, m, oa, ob, om = _twin(op2, 4096, 4096, 1, u, "m")
    x = op2.Dat(b, np.arange(4096, dtype=np.uint32), np.uint32, "x")
    ox = seq.Dat(ob, np.arange(4096, dtype=np.uint32), np.uint32)
    gp = b200.Plan(None, a, x(m[0], op2.WRITE), partition_size=128)
    ref = oplan.plan(oa, [ox(om[0], seq.WRITE)], partition_size=128)
    for name in ("nelems", "offset", "ind_map", "loc_map", "ind_sizes", "ind_offs", "nindirect"):
        np.testing.assert_array_equal(getattr(gp, name), getattr(ref, name), err_msg=name)
    assert gp.ncolors == 1 == ref.ncolors


def test_plan_matrix_coloring(op2):
    """test_coloring.py:84-114: Mat rows through elem_node (12 elements,
    random entries in [0, 4)) plus a WRITE Dat; partition 6."""
    from pyop2_b200 import b200
    rng = np.random.default_rng(3)
    vals = rng.integers(0, 4, size=(12, 3)).astype(np.int32)
    el, nd = op2.Set(12), op2.Set(36)
    m = op2.Map(el, nd, 3, vals, "elem_node")
    mat = op2.Mat(op2.Sparsity((m, m)), np.float64)
    x = op2.Dat(nd, np.zeros(36, dtype=np.uint32), np.uint32, "x")
    gp = b200.Plan(None, el, mat((m[op2.i[0]], m[op2.i[1]]), op2.INC), x(m[0], op2.WRITE),
                   partition_size=6, matrix_coloring=True)
    assert gp.nblocks == 2
    _check_thread_coloring(gp, 6, lambda e: vals[e])
    _check_block_coloring(gp, lambda blk: [vals[blk * 6:(blk + 1) * 6]])


def test_plan_large_random_validity(op2):
    from pyop2_b200 import b200
    rng = np.random.default_rng(0)
    n, nn = 200000, 50000
    vals = rng.integers(0, nn, size=(n, 2)).astype(np.int32)
    a, b = op2.Set(n), op2.Set(nn)
    m = op2.Map(a, b, 2, vals, "m")
    d = op2.Dat(b, np.zeros(nn), np.float64, "d")
    gp = b200.Plan(None, a, d(m[0], op2.INC), d(m[1], op2.INC), partition_size=512)
    _check_block_coloring(gp, lambda blk: [vals[blk * 512:(blk + 1) * 512]])
    thr, nth = gp.thrcol, gp.nthrcol
    for blk in range(0, gp.nblocks, 37):
        st, en = blk * 512, min(n, (blk + 1) * 512)
        for c in range(nth[blk]):
            rows = vals[st:en][thr[st:en] == c]
            flat = np.concatenate([np.unique(r) for r in rows]) if len(rows) else np.zeros(0)
            assert len(np.unique(flat)) == len(flat)


# --------------------------------------------------------------- sparsity
def _compare_sparsity(op2, rmult, cmult, pairs, nrows, ncols):
    """pairs: [(rvalues, cvalues, nelem, rarity, carity)] sharing row/col sets."""
    rows = op2.Set(nrows, rmult, "rows")
    cols = op2.Set(ncols, cmult, "cols")
    orows, ocols = seq.Set(nrows, rmult), seq.Set(ncols, cmult)
    gm, om = [], []
    for k, (rv, cv, ne, ra, ca) in enumerate(pairs):
        it, oit = op2.Set(ne), seq.Set(ne)
        gm.append((op2.Map(it, rows, ra, rv, "r%d" % k), op2.Map(it, cols, ca, cv, "c%d" % k)))
        om.append((seq.Map(oit, orows, ra, rv), seq.Map(oit, ocols, ca, cv)))
    sp = op2.Sparsity(tuple(gm) if len(gm) > 1 else gm[0])
    ref = seq.Sparsity(om)
    np.testing.assert_array_equal(sp._rowptr, ref.rowptr)
    np.testing.assert_array_equal(sp._colidx, ref.colidx)
    np.testing.assert_array_equal(sp._d_nnz, ref.nnz)
    from oracle import reference
    if reference.available():
        rr = seq.Sparsity(om, use_reference=True)
        np.testing.assert_array_equal(sp._rowptr, rr.rowptr)
        np.testing.assert_array_equal(sp._colidx, rr.colidx)
    return sp


def test_sparsity_random_maps(op2):
    rng = np.random.default_rng(5)
    ne, nn = 5000, 2000
    v = rng.integers(0, nn, size=(ne, 3)).astype(np.int32)
    _compare_sparsity(op2, 1, 1, [(v, v, ne, 3, 3)], nn, nn)


def test_sparsity_rectangular_and_vector(op2):
    rng = np.random.default_rng(6)
    ne = 3000
    rv = rng.integers(0, 700, size=(ne, 3)).astype(np.int32)
    cv = rng.integers(0, 900, size=(ne, 4)).astype(np.int32)
    _compare_sparsity(op2, 2, 3, [(rv, cv, ne, 3, 4)], 700, 900)


def test_sparsity_multiple_pairs(op2):
    rng = np.random.default_rng(8)
    a = rng.integers(0, 400, size=(1000, 3)).astype(np.int32)
    b = rng.integers(0, 400, size=(600, 2)).astype(np.int32)
    c = rng.integers(0, 500, size=(600, 2)).astype(np.int32)
    _compare_sparsity(op2, 1, 1, [(a, rng.integers(0, 500, size=(1000, 3)).astype(np.int32), 1000, 3, 3),
                                  (b, c, 600, 2, 2)], 400, 500)


def test_sparsity_high_degree_rows(op2):
    """Rows with more incidences than one warp keeps in shared memory."""
    rng = np.random.default_rng(9)
    ne = 20000
    v = rng.integers(0, 40, size=(ne, 3)).astype(np.int32)
    _compare_sparsity(op2, 1, 1, [(v, v, ne, 3, 3)], 40, 40)


def test_sparsity_p1_p2_meshes_nnz(op2):
    from pyop2_b200.workloads import meshes
    for n in (8, 64):
        c, e = meshes.square_p1(n)
        sp = _compare_sparsity(op2, 1, 1, [(e, e, len(e), 3, 3)], len(c), len(c))
        assert sp.nz == 7 * n * n + 6 * n + 1
        c, e = meshes.square_p2(n)
        sp = _compare_sparsity(op2, 1, 1, [(e, e, len(e), 6, 6)], len(c), len(c))
        assert sp.nz == 46 * n * n + 16 * n + 1


def test_sparsity_empty_rows(op2):
    v = np.array([[0, 2], [2, 4]], np.int32)
    sp = _compare_sparsity(op2, 1, 1, [(v, v, 2, 2, 2)], 6, 6)
    assert list(sp._d_nnz) == [2, 0, 3, 0, 2, 0]


# ------------------------------------------------- locality partition
def _region_check(op2, n, grow, stages, part, rs, inc=None, banks=False):
    """Device locality partition (op2b_region_plan_build) equals the numpy
    restatement (oracle/region.py) array for array; grow / stages are
    (values [n][arity], target size); inc flags the staged Maps the thread
    colours separate; banks applies the bank-aware slot numbering
    (op2b_region_plan_bank_slots) on both sides."""
    from oracle import region
    from pyop2_b200 import b200
    it = op2.Set(n)
    mk = {}

    def dmap(vals, ntg):
        key = id(vals)
        if key not in mk:
            mk[key] = op2.Map(it, op2.Set(ntg), vals.shape[1], vals)
        return mk[key]
    rp = b200.RegionPlan(n, part, rs, dmap(*grow), [dmap(v, t) for v, t in stages], inc,
                         bank_slots=banks)
    want = region.region_plan(grow[0], grow[1], [v for v, _ in stages], part, rs, inc)
    if banks:
        want = region.bank_slots(want, [v.shape[1] for v, _ in stages])
    for name in ("order", "boff", "tlist", "toff", "tcnt", "thrcol", "nthrcol"):
        np.testing.assert_array_equal(rp.host_array(name), want[name], err_msg=name)
    np.testing.assert_array_equal(rp.host_array("loc"), want["loc"].ravel())
    assert (rp.nregions, rp.levels) == (want["nregions"], want["levels"])
    ns = len(stages)
    nb = len(want["boff"]) - 1
    assert rp.nblocks == nb
    assert rp.max_count == [int(want["tcnt"][s::ns].max()) if nb else 0 for s in range(ns)]
    # blocks respect part_size and cover the set once
    assert (np.diff(want["boff"]) <= part).all()
    np.testing.assert_array_equal(np.sort(want["order"]), np.arange(n))
    return rp, want


@pytest.mark.parametrize("nx,ny,seed,part,rs,banks", [(60, 30, 0, 1024, 512, False),
                                                      (40, 17, 3, 256, 64, False),
                                                      (7, 5, 1, 32, 1000, False),
                                                      (60, 30, 0, 384, 192, True),
                                                      (7, 5, 1, 32, 1000, True)])
def test_region_plan_airfoil_matches_oracle(op2, nx, ny, seed, part, rs, banks):
    from pyop2_b200.workloads import meshes
    g = meshes.airfoil_grid(nx, ny, seed)
    pecell = np.asarray(g.pecell, np.int32).reshape(-1, 2)
    pedge = np.asarray(g.pedge, np.int32).reshape(-1, 2)
    rp, want = _region_check(op2, g.nedges, (pecell, g.ncells),
                             [(pecell, g.ncells), (pedge, g.nnodes)], part, rs, [True, False],
                             banks)
    assert rp.max_nthrcol == want["nthrcol"].max()
    if nx == 60:
        # compact regions: far fewer distinct cells per block than elements
        assert want["tcnt"][0::2].sum() < 0.7 * g.nedges


def test_region_plan_p2_and_disconnected(op2):
    from pyop2_b200.workloads import meshes
    coords, elem = meshes.square_p2(12, seed=4)
    elem = np.asarray(elem, np.int32)
    _region_check(op2, elem.shape[0], (elem, coords.shape[0]), [(elem, coords.shape[0])], 2048, 100)
    # arity 1 onto distinct targets: no element is adjacent to another, so
    # all but the seeds fall into the consecutive leftover regions
    n = 5000
    perm = np.random.default_rng(0).permutation(n).astype(np.int32).reshape(n, 1)
    _, want = _region_check(op2, n, (perm, n), [(perm, n)], 128, 64)
    assert want["levels"] == 1
    # empty set
    e = np.zeros((0, 2), np.int32)
    rp, _ = _region_check(op2, 0, (e, 4), [(e, 4)], 64, 64)
    assert rp.nblocks == 0
