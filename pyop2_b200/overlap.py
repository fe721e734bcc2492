"""Which par_loops of a captured step must follow which.

The reference runs every par_loop in program order (one stream, a
synchronise after each loop: pyop2/cuda.py:656-658).  A CUDA graph recorded
through :func:`pyop2_b200.b200.capture` keeps that order as a chain of nodes;
with overlap on, the chain edges between loops that touch no common data in
a conflicting way are dropped, so independent loops (airfoil: ``save_soln``
next to ``adt_calc``, ``bres_calc`` next to ``res_calc``) run side by side.

A segment is either a par_loop, given by its accesses -- ``(key, kind)``
pairs, ``key`` naming a Dat, Mat or Global, ``kind`` one of

* ``'R'``: read only;
* ``'I'``: increments added with atomic adds (indirect INC in the staged or
  atomic form, Mat INC in the atomic form), which commute with other such
  increments of the same object;
* ``'W'``: any other write (WRITE, RW, direct INC, Global reductions, the
  coloured and two-phase forms' plain read-modify-writes);

or ``None``: device work that is not a single par_loop launch (a copy, a
memset, a replica refresh, a loop with several launches).  ``None`` segments
are barriers: they follow everything before them and everything after them
follows them.

Rules per object: a read follows the last writers; a write follows the last
writers and every reader since; an atomic increment follows what the first
increment of its run followed (the writers and readers before the run), so
a run of increments to one object is unordered within itself.  Results
differ from program order only in the order of the commuting atomic adds,
which the atomic and staged forms leave unordered anyway.
"""


def loop_accesses(pairs):
    """Combine ``(key, kind)`` pairs of one loop: one kind per key, 'W' when
    a key appears with different kinds."""
    out = {}
    for key, kind in pairs:
        prev = out.get(key)
        out[key] = kind if prev is None or prev == kind else "W"
    return tuple(out.items())


def dependencies(segments, floating=None):
    """For each segment (accesses or None, in program order) the sorted list
    of earlier segments it must follow.

    ``floating`` (optional, one flag per segment): only the flagged loops
    are relaxed; every other loop also follows the previous unflagged loop
    (or barrier), so those keep program order among themselves.  The
    flagged ones are loops too small to fill the GPU, which then run beside
    their big neighbours instead of taking a turn of their own."""
    deps = _relaxed(segments)
    if floating is None:
        return deps
    out, prev = [], None
    for i, acc in enumerate(segments):
        d = set(deps[i])
        if acc is None:
            prev = i
        elif not floating[i]:
            if prev is not None:
                d.add(prev)
            prev = i
        out.append(sorted(d))
    return out


def _relaxed(segments):
    deps = []
    state = {}            # key -> {"w": writers, "r": readers, "inc": bool, "base": list}
    barrier = None
    since = []            # segments after the last barrier
    for i, acc in enumerate(segments):
        if acc is None:
            d = set(since)
            if barrier is not None:
                d.add(barrier)
            deps.append(sorted(d))
            barrier, since, state = i, [], {}
            continue
        d = set()
        if barrier is not None:
            d.add(barrier)
        for key, kind in acc:
            st = state.get(key)
            if st is None:
                st = state[key] = {"w": [], "r": [], "inc": False, "base": []}
            if kind == "R":
                d.update(st["w"])
                st["inc"] = False
                st["r"].append(i)
            elif kind == "I":
                if not st["inc"]:
                    st["base"] = st["w"] + st["r"]
                    st["w"], st["r"], st["inc"] = [], [], True
                d.update(st["base"])
                st["w"].append(i)
            elif kind == "W":
                d.update(st["w"])
                d.update(st["r"])
                st["w"], st["r"], st["inc"] = [i], [], False
            else:
                raise ValueError("access kind %r (R, I or W)" % (kind,))
        d.discard(i)
        deps.append(sorted(d))
        since.append(i)
    return deps
