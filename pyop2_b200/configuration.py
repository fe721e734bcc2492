"""OP2 configuration: a dict of defaults updated by ``op2.init(**kwargs)``.

Same keys as pyop2/assets/default.yaml (backend, debug, log_level) plus the
keys of the B200 backend:

* ``partition_size``: elements per plan block of indirect loops (default 0:
  chosen per loop by the backend);
* ``block_size``: threads per CTA of the generated stubs;
* ``fmad``: allow fused multiply-add contraction in JIT-compiled kernels
  (default False: every FP operation is rounded separately, like the host
  compiler on x86-64, so direct loops reproduce host results bit for bit);
* ``cache_dir``: directory of the on-disk cubin cache;
* ``validate_maps``: check Map values against their target Set on upload;
* ``l2_fetch_granularity``: per-context maximum L2 fetch granularity in bytes
  (32 suits gathers of small Dat rows through permuted Maps; 0 keeps the
  driver default);
* ``min_blocks_per_sm``: second __launch_bounds__ argument of the stubs (0:
  none), which caps registers per thread to raise occupancy;
* ``inc_mode``: how indirect loops resolve INC conflicts: ``'color'`` (plan
  with block and thread colouring; deterministic, bit-identical from run to
  run), ``'atomic'`` (one launch, atomic adds; summation order varies
  between runs within rounding) or ``'lma'`` (two phases: the stub stores
  every contribution, then each target adds its contributions in element
  order -- the sequential backend's order -- optionally Kahan-compensated;
  deterministic and independent of the launch configuration; loops it cannot
  run fall back to ``'color'``) or ``'staged'`` (one launch over a locality
  partition: the set is reordered into compact regions grown on the GPU,
  each block's distinct targets are staged in shared memory and INC rows
  accumulated there, then added once per target with atomics; summation
  order varies between runs within rounding; loops without indirect INC,
  with Mats, or whose staged rows would not fit a CTA's shared memory run
  as ``'atomic'``) or ``'gather'`` (loops whose only writes are INC into
  one Dat through one Map: one thread per target walks the target's
  incidence in element order, evaluates the kernel for each incident element
  and keeps its own share, then writes the target once -- no atomics, no
  colouring, the sequential backend's summation order; targets run in order
  of first use along the locality partition, so a warp's threads own
  neighbouring targets; other loops run as with ``'staged'``);
* ``region_size``: elements per region (one hashed seed per about this many
  elements) of the staged form's locality partition (0: half the partition
  size, whose default in the staged form is 384);
* ``staged_block_size``: threads per CTA of the staged form's stubs (one
  CTA per block of the partition);
* ``staged_tl_regs``: the staged stubs load their block's target ids into
  registers once (with the element rows) and reuse them for the row copies
  and the flush, which then adds one accumulated row per thread;
* ``staged_bank_slots``: renumber the staged rows of each block of the
  locality partition so that the rows eight neighbouring threads read lie in
  distinct shared-memory bank groups (``op2b_region_plan_bank_slots``);
* ``staged_pair``: 2 makes each thread of a staged stub evaluate two
  elements (of two consecutive passes) before one shared run of colour
  rounds; 1 (default) one element per pass;
* ``direct_unroll``: elements each thread of a direct stub takes per round
  (their rows all loaded before the kernel calls, so the loads overlap);
* ``staged_min_size``: iteration sets smaller than this run the atomic form
  even when ``inc_mode`` is ``'staged'`` (a partition of them has too few
  blocks to fill the GPU);
* ``owner_mode``: owner-computes for loops whose only write is INC into one
  Dat through one Map or into one scalar Mat: one warp per target adds the
  target's contributions in the sequential backend's order and writes it once
  (deterministic, no atomics, bit-identical to the sequential backend's
  order).  ``'auto'`` uses it for Mats and 1-d iteration-space INC (no
  redundant kernel evaluation), ``'always'`` also for vec-map / indexed INC,
  ``'never'`` (default) leaves those loops to ``inc_mode``.  It is slower than
  the atomic form where kernels index tables with the iteration-space index
  (the index becomes a run-time value per lane);
* ``kahan``: compensated (Kahan) summation of owner-computes and two-phase
  (``inc_mode='lma'``) accumulation;
* ``mat_slots``: assemble scalar Mats in the atomic form through a cached
  scatter-slot table (the CSR position of every element's local entries,
  built once per Sparsity and Map pair: nelem x arity^2 int32 of device
  memory) instead of searching the CSR row for every entry;
* ``mat_per_entry``: with slot tables, add each scalar Mat entry right after
  the kernel call that computed it instead of after the whole local tensor
  (one entry live in registers instead of the tensor; Mats on one Sparsity
  through one Map pair share one slot load);
* ``read_replicas``: a loop of the atomic form (no plan, elements in set
  order) on a set of at least ``replica_min_size`` elements that only reads
  a Dat through a Map reads a device copy of the Dat kept in order of first
  use through that Map, through the Map renumbered to match: rows
  neighbouring elements read lie next to each other.  The copy is refreshed
  when the Dat was written since (host writes, loops, zero, arithmetic);
  it costs one extra copy of the Dat and of the Map;
* ``gathered_replicas``: with ``read_replicas``, such a loop reads the Dat
  from a copy gathered element by element (row k of element e at
  e * arity + k: no Map read, no dependent gather) when that copy takes at
  most ``gathered_max_gb`` GB (arity copies of each row);
* ``fmad_inc``: compile the element code of loops with indirect INC in the
  staged, atomic, gather and coloured forms with multiply-add contraction
  (their sums are reassociated anyway, so they already differ from the
  sequential order within rounding); other loops keep ``fmad``;
* ``programmatic_launch``: launch the generated stubs with programmatic
  stream serialisation, so a stub's CTAs are scheduled while the kernel
  before it drains (each stub waits for that kernel's completion before it
  touches memory);
* ``itspace_split``: ``'RxC'`` (e.g. ``'2x2'``) splits the 2-d iteration
  space of an atomic-form Mat assembly (scalar Mats added entry by entry,
  every other argument READ) into R x C blocks of local positions evaluated
  by different warps for the same 32 elements: fewer values live per
  thread, more warps resident; ``''`` keeps one thread per element;
  ``'auto'`` (default) splits 3 x 2 when the local block has at least 36
  entries (P2 and up) and keeps one thread per element below;
* ``mat_slots_rel``: with per-entry adds, read each local row's columns
  from a compact slot table (one 64-bit word of in-row positions per element
  and local row, added to the row start read through the Map) instead of one
  32-bit position per local entry;
* ``graph_overlap``: a CUDA graph recorded with ``b200.capture`` lets
  par_loops that touch no common data in a conflicting way run side by side
  (reads of one object, atomic increments of one object): ``True`` every
  such loop, ``'small'`` only loops over fewer elements than one 256-thread
  CTA per SM covers (they run beside their big neighbours, which keep
  program order among themselves), ``False`` none; other device work
  recorded in the graph stays in program order with everything around it;
* ``hbm_budget_gb``: device memory (GB) the serving engine's MeshStore
  admits meshes and requests against by default;
* ``pool_reserve_gb``: device memory (GB, at most a quarter of the device)
  the stream-ordered allocation pool is grown to at initialisation; freed
  memory stays in the pool, so allocations up to this size never map fresh
  device memory later (0: grow on demand).
"""

import os

_defaults = {
    'backend': 'b200',
    'debug': 0,
    'log_level': 'WARN',
    'python_plan': True,
    'partition_size': 0,
    'block_size': 256,
    'fmad': False,
    'cache_dir': os.environ.get('OP2B_CACHE_DIR',
                                os.path.join('/tmp', 'op2b200-cache-%d' % os.getuid())),
    'validate_maps': True,
    'device': 0,
    'l2_fetch_granularity': 32,
    'min_blocks_per_sm': 0,
    'inc_mode': 'staged',
    'region_size': 0,
    'staged_min_size': 262144,
    'staged_block_size': 128,
    'owner_mode': 'never',
    'kahan': False,
    'mat_slots': True,
    'mat_per_entry': True,
    'read_replicas': True,
    'replica_min_size': 262144,
    'gathered_replicas': False,
    'gathered_max_gb': 2.0,
    'fmad_inc': False,
    'programmatic_launch': False,
    'itspace_split': 'auto',
    'staged_tl_regs': False,
    'direct_unroll': 1,
    'mat_slots_rel': False,
    'graph_overlap': False,
    'staged_pair': 1,
    'staged_bank_slots': False,
    'hbm_budget_gb': 120.0,
    'pool_reserve_gb': 4.0,
}

_config = dict(_defaults)


_generation = [0]


def generation():
    """Changes whenever the configuration may have changed (cache keys)."""
    return _generation[0]


def configure(**kwargs):
    for k, v in kwargs.items():
        if k == 'log_level' and v is None:
            continue
        _config[k] = v
    _generation[0] += 1


def reset():
    _config.clear()
    _config.update(_defaults)
    _generation[0] += 1


def __getitem__(key):  # pragma: no cover - module-level item access shim
    return _config[key]


def get(key, default=None):
    return _config.get(key, default)


class _ConfigView(object):
    def __getitem__(self, key):
        return _config[key]

    def __getattr__(self, key):
        try:
            return _config[key]
        except KeyError:
            raise AttributeError(key)


cfg = _ConfigView()
