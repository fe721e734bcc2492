"""The locality-partition restatement (oracle/region.py) checked against
the properties the staged form relies on, so the checker of the device
builder is itself checked: the order is a permutation, blocks respect the
partition size, every block's staged list holds exactly its elements'
targets in first-use order and loc points into it, thread colours separate
the INC targets, and positions are sorted by colour within a block.  CPU
only."""

import numpy as np
import pytest

from oracle import region
from pyop2_b200.workloads import meshes


def _check(grow, ntargets, stages, part, rs, inc):
    n = grow.shape[0]
    R = region.region_plan(grow, ntargets, stages, part, rs, inc)
    order, boff = R["order"], R["boff"]
    np.testing.assert_array_equal(np.sort(order), np.arange(n))
    assert boff[0] == 0 and boff[-1] == n and (np.diff(boff) > 0).all() and (np.diff(boff) <= part).all()
    ns = len(stages)
    row = 0
    rows = []
    for v in stages:
        rows.append(row)
        row += v.shape[1]
    for b in range(len(boff) - 1):
        seg = slice(boff[b], boff[b + 1])
        el = order[seg]
        for s, v in enumerate(stages):
            lo, cnt = R["toff"][b * ns + s], R["tcnt"][b * ns + s]
            tl = R["tlist"][lo:lo + cnt]
            assert len(set(tl.tolist())) == cnt
            assert set(tl.tolist()) == set(v[el].ravel().tolist())
            for r in range(v.shape[1]):
                np.testing.assert_array_equal(tl[R["loc"][rows[s] + r, seg]], v[el, r])
        col = R["thrcol"][seg]
        assert (np.diff(col) >= 0).all() and R["nthrcol"][b] == col.max() + 1
        for c in range(R["nthrcol"][b]):
            for s, v in enumerate(stages):
                if inc[s]:
                    t = [tuple(sorted(set(x))) for x in v[el[col == c]].tolist()]
                    flat = [x for tt in t for x in tt]
                    assert len(flat) == len(set(flat)), "colour %d shares a target" % c
    return R


def test_airfoil_partition_properties_and_locality():
    g = meshes.airfoil_grid(40, 20, 4)
    pc = np.asarray(g.pecell, np.int32).reshape(-1, 2)
    pe = np.asarray(g.pedge, np.int32).reshape(-1, 2)
    R = _check(pc, g.ncells, [pc, pe], 384, 192, [True, False])
    # compact regions on a permuted mesh: far fewer distinct cells per edge
    # than the 1.3 of consecutive blocks
    assert R["tcnt"][0::2].sum() / pc.shape[0] < 0.7


@pytest.mark.parametrize("seed", [0, 1])
def test_random_graph_and_degenerate_rows(seed):
    rng = np.random.default_rng(seed)
    m = rng.integers(0, 500, size=(3000, 3)).astype(np.int32)
    m[::13, 2] = m[::13, 0]                     # an element touching one target twice
    _check(m, 500, [m], 128, 64, [True])


def test_p2_first_use_numbering():
    coords, elem = meshes.square_p2(10, seed=2)
    elem = np.asarray(elem, np.int32)
    _check(elem, coords.shape[0], [elem], 256, 128, [True])
    # first use: walking a block's positions (rows in order), each target's
    # number is the count of distinct targets seen before it.  Numbers are
    # given before positions are sorted by colour, so the walk is checked
    # without INC targets (one colour, nothing moves)
    R = _check(elem, coords.shape[0], [elem], 256, 128, [False])
    b0 = slice(R["boff"][0], R["boff"][1])
    loc = R["loc"][:, b0].T.ravel()
    seen = []
    for x in loc:
        if x not in seen:
            assert x == len(seen)
            seen.append(x)


def test_single_seed_and_empty():
    m = np.arange(10, dtype=np.int32).reshape(10, 1)
    R = _check(m, 10, [m], 4, 100, [True])      # element 0 is always a seed
    assert R["levels"] == 1
    e = np.zeros((0, 2), np.int32)
    R = region.region_plan(e, 4, [e], 64, 64)
    assert len(R["boff"]) == 1 and R["order"].size == 0


def test_bank_slots_keep_targets_and_cut_conflicts():
    """The bank-aware slot numbering (restated in oracle/region.py, the
    checker of op2b_region_plan_bank_slots) keeps every (position, row)'s
    target, marks padding slots -1, and removes a part of the bank-group conflicts of
    the staged-row reads on the airfoil edges."""
    g = meshes.airfoil_grid(60, 30, 0)
    pecell = np.asarray(g.pecell, np.int64).reshape(-1, 2)
    pedge = np.asarray(g.pedge, np.int64).reshape(-1, 2)
    stages = [pecell, pedge]
    R = region.region_plan(pecell, g.ncells, stages, 384, 192, [True, False])
    B = region.bank_slots(R, [2, 2])
    ns, n = 2, g.nedges
    for k in ("order", "boff", "thrcol", "nthrcol"):
        np.testing.assert_array_equal(B[k], R[k])
    for b in range(len(R["boff"]) - 1):
        seg = slice(R["boff"][b], R["boff"][b + 1])
        for s, v in enumerate(stages):
            lo, cnt = B["toff"][b * ns + s], B["tcnt"][b * ns + s]
            tl = B["tlist"][lo:lo + cnt]
            real = tl[tl >= 0]
            assert sorted(real.tolist()) == sorted(set(v[R["order"][seg]].ravel().tolist()))
            for r in range(2):
                np.testing.assert_array_equal(tl[B["loc"][2 * s + r, seg]], v[R["order"][seg], r])
            # at most one residue class longer than the others by the balance rule
            assert cnt <= 8 * (-(-R["tcnt"][b * ns + s] // 8)) + 8 * 4
    before = region.bank_conflicts(R, [2, 2], 2)
    after = region.bank_conflicts(B, [2, 2], 2)
    assert after < 0.8 * before, (before, after)
    assert n == R["loc"].shape[1]
