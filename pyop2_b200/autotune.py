"""Launch-configuration autotuner for batched loops.

For a batch of loop instances (one signature) the tuner times each candidate
configuration -- the colouring granularity (element-level atomics, or the
coloured form: each mesh partitioned into blocks of ``part_size`` elements
with block and thread colours, pyop2/plan.pyx:214-376), the partition size
(``part_size`` of the coloured form; threads per CTA x elements per thread,
the tile handed to one CTA, of the atomic form), threads per CTA (block
shape), the stub's minimum resident CTAs per SM (register cap) and the
persistent grid's CTAs per SM -- on the batch itself, with CUDA events after one untimed launch, and keeps the
fastest.  Results are cached in memory and in ``<cache_dir>/autotune.json``
under a key made of the loop signature and the batch's size class, so a
served or repeated batch of the same kind is not re-tuned.

There is no counterpart in the reference (pyop2/cuda.py fixed the block size
at 128 and derived the partition size from shared memory,
pyop2/cuda.py:660-700).
"""

import hashlib
import json
import os
import statistics

from . import b200
from . import configuration as cfg

DEFAULT_CANDIDATES = tuple(
    dict(block_size=bs, elems_per_thread=ept, min_blocks=mb, ctas_per_sm=0)
    for bs in (128, 256, 512) for ept in (1, 2, 4) for mb in (0,))

# The coloured form's candidates: partition size (elements per block of each
# instance's plan) x threads per CTA; the colouring granularity is the
# choice between these and the element-level atomics above.
COLOURED_CANDIDATES = tuple(
    dict(form="color", part_size=ps, block_size=bs, min_blocks=0, ctas_per_sm=0)
    for ps in (128, 512) for bs in (128, 256) if bs <= ps)


def candidates_for(instances):
    """The search space of a batch: atomic launch shapes, plus the coloured
    form's partition sizes where the loop has indirect INC (a plan applies)
    and no Global reduction."""
    spec = instances[0].spec
    out = list(DEFAULT_CANDIDATES)
    if spec.mode == "atomic" and instances[0].form == "atomic" and not any(
            a.kind == "gbl" and a.access != "READ" for a in spec.args):
        out += list(COLOURED_CANDIDATES)
    return tuple(out)

_MEM = {}


def _path():
    return os.path.join(cfg.cfg['cache_dir'], "autotune.json")


def _load():
    try:
        with open(_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(key, entry):
    d = _load()
    d[key] = entry
    try:
        os.makedirs(cfg.cfg['cache_dir'], exist_ok=True)
        tmp = _path() + ".%d.tmp" % os.getpid()
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, _path())
    except OSError:
        pass


def size_class(elements, segments):
    """Batches within a factor of two in total elements and in segment count
    share a tuning result."""
    return (max(0, int(elements)).bit_length(), max(0, int(segments)).bit_length())


def tuning_key(instances):
    sig = repr(instances[0].key).encode()
    elems = sum(i.size for i in instances)
    return "%s:%d:%d" % ((hashlib.sha256(sig).hexdigest()[:24],) + size_class(elems, len(instances)))


def time_launch(runner, reps=3, flush=True, before=None):
    """Median device time (ms) of runner.launch() over reps, after one
    untimed launch; L2 flushed and ``before()`` (untimed) run before each
    timed launch."""
    if before is not None:
        before()
    runner.launch()
    b200.synchronize()
    ts = []
    for _ in range(reps):
        if before is not None:
            before()
        if flush:
            b200.l2_flush()
        e0 = b200.Event().record()
        runner.launch()
        e1 = b200.Event().record()
        e1.synchronize()
        ts.append(e0.elapsed_ms(e1))
    return statistics.median(ts)


def tune(instances, candidates=None, reps=3, use_cache=True, restore=None):
    """Best BatchLoop configuration for ``instances``: returns (config dict,
    {config repr: ms}).  Candidates with ``form='color'`` run the coloured
    form (the instances recast with a plan of ``part_size`` elements per
    block); the others the atomic form.  Each timed launch really runs the
    loops, so INC targets accumulate: ``restore`` (a callable, untimed) is
    invoked before every launch if the caller needs the data reset (e.g.
    zeroing Mats)."""
    from .batch import BatchLoop
    if candidates is None:
        candidates = candidates_for(instances)
    key = tuning_key(instances)
    if use_cache:
        hit = _MEM.get(key) or _load().get(key)
        if hit:
            _MEM[key] = hit
            return dict(hit["best"]), hit.get("times", {})
    times = {}
    best, best_ms = None, None

    class _Runner(object):
        def __init__(self, bl):
            self.bl = bl

        def launch(self):
            self.bl.launch(sync_host=False)

    recast = {}
    for c in candidates:
        c = dict(c)
        form = c.pop("form", "atomic")
        ps = c.pop("part_size", None)
        if form == "color":
            if ps not in recast:
                try:
                    recast[ps] = [i.recast("color", ps) for i in instances]
                except NotImplementedError:
                    recast[ps] = None
            if recast[ps] is None:
                continue
            bl = BatchLoop(recast[ps], **c)
        else:
            bl = BatchLoop(instances, **c)
        ms = time_launch(_Runner(bl), reps=reps, before=restore)
        if form == "color":
            c = dict(c, form=form, part_size=ps)
        times[json.dumps(c, sort_keys=True)] = round(ms, 5)
        if best_ms is None or ms < best_ms:
            best, best_ms = dict(c), ms
        del bl
    entry = {"best": best, "ms": best_ms, "times": times}
    _MEM[key] = entry
    if use_cache:
        _store(key, entry)
    return dict(best), times


def build(instances, config):
    """A BatchLoop over ``instances`` in the form and shape ``config`` names
    (a tuning result)."""
    from .batch import BatchLoop
    c = dict(config)
    form = c.pop("form", "atomic")
    ps = c.pop("part_size", None)
    if form == "color":
        instances = [i.recast("color", ps) for i in instances]
    return BatchLoop(instances, **c)


def tuned_batch(instances, **kw):
    """A BatchLoop over ``instances`` with the tuned configuration."""
    best, _ = tune(instances, **kw)
    return build(instances, best)
