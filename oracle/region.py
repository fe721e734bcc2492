"""Test infrastructure: CPU restatement (numpy) of the locality partition the
B200 backend builds on the GPU for its staged indirect loops
(op2b_region_plan_build), used only by tests as the checker.

The reference has no such structure: it partitions an iteration set into
blocks of consecutive elements (pyop2/plan.pyx:107-110) and stages each
block's indirect rows (:112-212).  The staged loops' results are checked
against the sequential oracle (oracle/seq.py); this module pins the
partition itself, which is deterministic, so the device arrays must equal
these bit for bit:

* seeds: element 0 and every element whose 32-bit hash is divisible by
  region_size; region id = rank of the seed;
* multi-source breadth-first search over the elements, two elements being
  adjacent when they share a value of the growth Map; an element reached at
  level L+1 takes the smallest (level, region) key among its targets, which
  carry the key of the smallest level-L element touching them;
* elements not reached form regions nseeds + e // part_size at level 0;
* order: elements sorted by (region, level, element id) (level dropped from
  the key when regions x levels exceeds max(4 n, 2^20));
* blocks: each region cut into ceil(size / part_size) runs, boundaries at
  start + size * q // pieces;
* staging: per block and staged Map the distinct values over all rows,
  numbered in order of first use (positions in order, each position's rows
  in order), and each (position, row)'s number;
* thread colours: per block, elements in position order take the lowest
  colour (of 32 per round) that no earlier element sharing one of its INC
  staged targets holds (pyop2/plan.pyx:282-324); then the block's positions
  are sorted by colour (stable): order, loc and thrcol follow.
"""

import numpy as np

UNSET = np.iinfo(np.uint64).max


def _hash(x):
    x = x.astype(np.uint64)
    m = np.uint64(0xFFFFFFFF)
    x ^= x >> np.uint64(16)
    x = (x * np.uint64(0x7FEB352D)) & m
    x ^= x >> np.uint64(15)
    x = (x * np.uint64(0x846CA68B)) & m
    x ^= x >> np.uint64(16)
    return x


def regions(grow_values, ntargets, region_size):
    """Per element key (level << 32 | region) or UNSET, number of seeds,
    deepest level."""
    gm = np.asarray(grow_values, dtype=np.int64)
    n = gm.shape[0]
    e = np.arange(n)
    seed = (_hash(e) % np.uint64(region_size)) == 0
    if n:
        seed[0] = True
    rank = np.cumsum(seed) - seed
    ekey = np.where(seed, rank.astype(np.uint64), UNSET).astype(np.uint64)
    tkey = np.full(ntargets, UNSET, dtype=np.uint64)
    level = 0
    levels = 0
    while n:
        act = (ekey != UNSET) & ((ekey >> np.uint64(32)) == np.uint64(level))
        for r in range(gm.shape[1]):
            np.minimum.at(tkey, gm[act, r], ekey[act])
        un = ekey == UNSET
        best = tkey[gm[:, 0]].copy()
        for r in range(1, gm.shape[1]):
            best = np.minimum(best, tkey[gm[:, r]])
        new = un & (best != UNSET)
        if not new.any():
            break
        ekey[new] = (((best[new] >> np.uint64(32)) + np.uint64(1)) << np.uint64(32)) | \
            (best[new] & np.uint64(0xFFFFFFFF))
        level += 1
        levels = level
    return ekey, int(seed.sum()), levels


def _thread_colors(targets):
    """Greedy colouring of one block; targets[i] = the INC targets of the
    block's i-th element."""
    col = [-1] * len(targets)
    base, remaining = 0, len(targets)
    while remaining:
        masks = {}
        remaining = 0
        for i, ts in enumerate(targets):
            if col[i] >= 0:
                continue
            m = 0
            for t in ts:
                m |= masks.get(t, 0)
            if m == 0xFFFFFFFF:
                remaining += 1
                continue
            c = (~m & (m + 1)).bit_length() - 1
            col[i] = base + c
            for t in ts:
                masks[t] = masks.get(t, 0) | (1 << c)
        base += 32
    return col


def region_plan(grow_values, ntargets, stage_values, part_size, region_size, stage_inc=None):
    """Returns dict(order, boff, tlist, toff, tcnt, loc, thrcol, nthrcol,
    nregions, levels) in the device layout (loc: [sum of arities][n]
    int16); stage_inc flags the staged Maps whose targets the thread colours
    separate (default all)."""
    ekey, nseeds, levels = regions(grow_values, ntargets, region_size)
    n = ekey.shape[0]
    e = np.arange(n, dtype=np.int64)
    nregions = nseeds + -(-max(n, 1) // part_size)
    unset = ekey == UNSET
    region = np.where(unset, nseeds + e // part_size, (ekey & np.uint64(0xFFFFFFFF)).astype(np.int64))
    level = np.where(unset, 0, (ekey >> np.uint64(32)).astype(np.int64))
    nlevels = levels + 1
    if nregions * nlevels > max(4 * n, 1 << 20) or nregions * nlevels >= 2 ** 31 - 1:
        nlevels = 1
    bucket = region * nlevels + (level if nlevels > 1 else 0)
    order = np.lexsort((e, bucket)).astype(np.int32)
    sizes = np.bincount(region, minlength=nregions)
    starts = np.concatenate([[0], np.cumsum(sizes)])
    boff = [0]
    for r in range(nregions):
        cnt = int(sizes[r])
        if cnt <= 0:
            continue
        pieces = -(-cnt // part_size)
        for q in range(1, pieces + 1):
            boff.append(int(starts[r]) + cnt * q // pieces)
    boff = np.asarray(boff, dtype=np.int32)
    nb = len(boff) - 1
    stage_values = [np.asarray(v, dtype=np.int64) for v in stage_values]
    stage_values = [v if v.ndim == 2 else v.reshape(n, -1) for v in stage_values]
    ns = len(stage_values)
    tcnt = np.zeros(nb * ns, dtype=np.int32)
    lists = []
    rows = sum(v.shape[1] for v in stage_values)
    loc = np.zeros((rows, n), dtype=np.int16)
    for b in range(nb):
        el = order[boff[b]:boff[b + 1]]
        row = 0
        for s, v in enumerate(stage_values):
            flat = v[el].ravel()
            u, first, inv = np.unique(flat, return_index=True, return_inverse=True)
            rank = np.argsort(first, kind="stable")
            num = np.empty_like(rank)
            num[rank] = np.arange(rank.size)
            tcnt[b * ns + s] = u.size
            lists.append(u[rank])
            loc[row:row + v.shape[1], boff[b]:boff[b + 1]] = num[inv].reshape(-1, v.shape[1]).T
            row += v.shape[1]
    toff = np.concatenate([[0], np.cumsum(tcnt)]).astype(np.int32)
    tlist = np.concatenate(lists).astype(np.int32) if lists else np.zeros(0, np.int32)
    inc = [True] * ns if stage_inc is None else list(stage_inc)
    thrcol = np.zeros(n, dtype=np.int32)
    nthrcol = np.zeros(nb, dtype=np.int32)
    for b in range(nb):
        el = order[boff[b]:boff[b + 1]]
        targets = [[(s, int(t)) for s, v in enumerate(stage_values) if inc[s] for t in v[i]]
                   for i in el]
        col = np.asarray(_thread_colors(targets), dtype=np.int32)
        perm = np.argsort(col, kind="stable")
        seg = slice(boff[b], boff[b + 1])
        thrcol[seg] = col[perm]
        order[seg] = order[seg][perm]
        loc[:, seg] = loc[:, seg][:, perm]
        nthrcol[b] = col.max() + 1 if col.size else 0
    return dict(order=order, boff=boff, tlist=tlist, toff=toff, tcnt=tcnt, loc=loc,
                thrcol=thrcol, nthrcol=nthrcol, nregions=nregions, levels=levels + 1)


def bank_slots(plan, arities):
    """The plan with its staged slots renumbered for shared-memory bank
    groups, as op2b_region_plan_bank_slots does: per (block, staged Map),
    over groups of 8 consecutive positions and row by row, every target not
    yet placed takes the residue mod 8 unused in its group with the fewest
    targets so far (ties: the lowest residue; any residue when all 8 are
    used); slots are residue + 8 * rank in the residue class (first-use
    order); padding slots hold target -1."""
    boff, tcnt, toff, tlist, loc = (plan[k] for k in ("boff", "tcnt", "toff", "tlist", "loc"))
    ns, nb = len(arities), len(boff) - 1
    row0 = np.concatenate([[0], np.cumsum(arities)]).astype(np.int64)
    new_loc = loc.copy()
    ncnt = np.zeros(nb * ns, dtype=np.int32)
    lists = []
    for b in range(nb):
        start, nelem = int(boff[b]), int(boff[b + 1] - boff[b])
        for s in range(ns):
            nu = int(tcnt[b * ns + s])
            res = [-1] * nu
            cls = [0] * 8
            for g in range(0, nelem, 8):
                m = min(8, nelem - g)
                for r in range(arities[s]):
                    ts = [int(loc[row0[s] + r, start + g + i]) for i in range(m)]
                    used = 0
                    for t in ts:
                        if res[t] >= 0:
                            used |= 1 << res[t]
                    for t in ts:
                        if res[t] >= 0:
                            continue
                        free = 0xFF if used == 0xFF else (~used & 0xFF)
                        best = -1
                        for c in range(8):
                            if (free >> c) & 1 and (best < 0 or cls[c] < cls[best]):
                                best = c
                        res[t] = best
                        cls[best] += 1
                        used |= 1 << best
            nxt = [0] * 8
            perm = np.zeros(nu, dtype=np.int64)
            for k in range(nu):
                c = max(res[k], 0)
                perm[k] = c + 8 * nxt[c]
                nxt[c] += 1
            top = int(perm.max()) + 1 if nu else 0
            ncnt[b * ns + s] = top
            lst = np.full(top, -1, dtype=np.int32)
            lst[perm] = tlist[toff[b * ns + s]:toff[b * ns + s] + nu]
            lists.append(lst)
            for r in range(arities[s]):
                seg = new_loc[row0[s] + r, start:start + nelem]
                new_loc[row0[s] + r, start:start + nelem] = perm[seg.astype(np.int64)]
    out = dict(plan)
    out.update(tcnt=ncnt, toff=np.concatenate([[0], np.cumsum(ncnt)]).astype(np.int32),
               tlist=np.concatenate(lists).astype(np.int32) if lists else np.zeros(0, np.int32),
               loc=new_loc)
    return out


def bank_conflicts(plan, arities, chunks):
    """Extra 16-byte bank-group wavefronts of the staged-row reads of a
    plan: per group of 8 consecutive positions of a block and per row, the
    largest number of distinct slots sharing a residue mod 8, minus one,
    summed; ``chunks`` is the row size in 16-byte chunks (informative
    metric for tests)."""
    boff, loc = plan["boff"], plan["loc"]
    row0 = np.concatenate([[0], np.cumsum(arities)]).astype(np.int64)
    total = 0
    for b in range(len(boff) - 1):
        start, nelem = int(boff[b]), int(boff[b + 1] - boff[b])
        for s in range(len(arities)):
            for g in range(0, nelem, 8):
                m = min(8, nelem - g)
                for r in range(arities[s]):
                    slots = set(int(x) for x in loc[row0[s] + r, start + g:start + g + m])
                    counts = np.bincount([x % 8 for x in slots], minlength=8)
                    total += (int(counts.max()) - 1) * chunks
    return total
