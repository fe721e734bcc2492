"""Dependencies between the par_loops of an overlapped capture
(pyop2_b200/overlap.py): pure host logic, no GPU.

The reference runs loops in program order (pyop2/cuda.py:656-658); an
overlapped graph may only drop an order between two loops when neither
reads what the other writes, or both only add atomically to it."""

import pytest

from pyop2_b200 import overlap


def _airfoil_step():
    """The accesses of one airfoil iteration (pyop2/demo/airfoil.py:88-131)
    as the B200 forms classify them: res_calc staged and bres_calc atomic add
    to res with atomics; update writes q and res and reduces rms."""
    save = (("q", "R"), ("qold", "W"))
    adt = (("x", "R"), ("q", "R"), ("adt", "W"))
    res = (("x", "R"), ("q", "R"), ("adt", "R"), ("res", "I"))
    bres = (("x", "R"), ("q", "R"), ("adt", "R"), ("res", "I"), ("bound", "R"))
    upd = (("qold", "R"), ("q", "W"), ("res", "W"), ("adt", "R"), ("rms", "W"))
    return [save, adt, res, bres, upd, adt, res, bres, upd]


def test_airfoil_step():
    d = overlap.dependencies(_airfoil_step())
    assert d[0] == []
    assert d[1] == []                      # adt_calc next to save_soln
    assert d[2] == [1]                     # res_calc after adt_calc
    assert d[3] == [1]                     # bres_calc next to res_calc
    assert d[4] == [0, 1, 2, 3]            # update after everything
    assert d[5] == [1, 2, 3, 4]            # adt_calc after update (q) and its readers of adt
    assert d[6] == [4, 5]
    assert d[7] == [4, 5]
    assert d[8] == [0, 4, 5, 6, 7]


def test_every_conflict_is_ordered():
    """Brute force over random access lists: two loops that touch one key,
    one of them writing it (other than two atomic adds), are ordered by the
    transitive closure of the dependencies."""
    import random
    rnd = random.Random(7)
    for _ in range(300):
        n = rnd.randint(1, 12)
        segs = []
        for _ in range(n):
            if rnd.random() < 0.1:
                segs.append(None)
                continue
            segs.append(overlap.loop_accesses(
                [(rnd.choice("abcd"), rnd.choice("RIW")) for _ in range(rnd.randint(1, 3))]))
        deps = overlap.dependencies(segs)
        before = [set() for _ in range(n)]
        for i in range(n):
            for j in deps[i]:
                assert j < i
                before[i] |= {j} | before[j]
        for i in range(n):
            for j in range(i):
                if segs[i] is None or segs[j] is None:
                    assert j in before[i]
                    continue
                a, b = dict(segs[j]), dict(segs[i])
                for key in set(a) & set(b):
                    ka, kb = a[key], b[key]
                    if ka == "R" and kb == "R" or ka == "I" and kb == "I":
                        continue
                    assert j in before[i], (segs, deps, i, j, key)


def test_atomic_runs_are_unordered():
    inc = (("res", "I"),)
    d = overlap.dependencies([(("res", "W"),), inc, inc, inc, (("res", "R"),), inc])
    assert d[1] == d[2] == d[3] == [0]
    assert d[4] == [1, 2, 3]
    assert d[5] == [1, 2, 3, 4]            # a new run follows the read


def test_barriers():
    r = (("x", "R"),)
    d = overlap.dependencies([r, r, None, r, r, None])
    assert d == [[], [], [0, 1], [2], [2], [2, 3, 4]]


def test_mixed_kinds_of_one_key_write():
    assert dict(overlap.loop_accesses([("a", "R"), ("a", "I")]))["a"] == "W"
    assert dict(overlap.loop_accesses([("a", "I"), ("a", "I")]))["a"] == "I"
    with pytest.raises(ValueError):
        overlap.dependencies([(("a", "X"),)])


def test_airfoil_step_small_loops_float():
    """Only bres_calc (3,600 edges) floats: it runs beside res_calc, while
    the big loops keep program order among themselves."""
    fl = [False, False, False, True, False, False, False, True, False]
    d = overlap.dependencies(_airfoil_step(), fl)
    assert d[1] == [0]                     # adt_calc after save_soln (both big)
    assert d[2] == [1]
    assert d[3] == [1]                     # bres_calc beside res_calc
    assert d[4] == [0, 1, 2, 3]            # update waits for both
    assert d[5] == [1, 2, 3, 4]
    assert d[7] == [4, 5]                  # the second bres_calc beside the second res_calc
    assert d[8] == [0, 4, 5, 6, 7]
    # nothing floats: program order
    chain = overlap.dependencies(_airfoil_step(), [False] * 9)
    assert all(i - 1 in chain[i] for i in range(1, 9))


def test_floating_loops_keep_every_conflict_ordered():
    """A floating loop still follows every conflicting earlier loop, and a
    barrier orders everything around it."""
    segs = [(("a", "W"),), (("b", "W"),), None, (("a", "R"),), (("c", "W"),)]
    d = overlap.dependencies(segs, [False, True, False, True, False])
    assert d[1] == []                      # floats: no conflict with segment 0
    assert d[2] == [0, 1]                  # barrier after both
    assert d[3] == [2]                     # after the barrier only
    assert d[4] == [2]                     # big loop: after the barrier (previous big)


def test_capture_modes():
    """b200.capture(overlap=...) accepts True, False and 'small' (the
    configuration key's values) and nothing else; no device is touched
    before the block is entered."""
    from pyop2_b200 import b200
    assert (b200.capture(overlap=True).overlap, b200.capture(overlap=True).small_only) == (True, False)
    assert (b200.capture(overlap="small").overlap, b200.capture(overlap="small").small_only) == (True, True)
    assert b200.capture(overlap=False).overlap is False
    with pytest.raises(ValueError):
        b200.capture(overlap="sometimes")
