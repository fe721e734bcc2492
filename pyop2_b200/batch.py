"""Batched par_loops: one loop signature over many independent instances.

A :class:`LoopInstance` is one par_loop (a kernel, an iteration set and its
arguments) whose objects stay resident on the device.  A :class:`BatchLoop`
runs any number of instances that share a loop signature (same kernel, same
argument kinds, types, arities and access modes; different Sets, Maps, Dats,
Mats and Globals) in ONE persistent launch:

* every instance is a *segment*; its parameter block (the same
  ``op2b_params`` struct a single par_loop passes by value) is packed once, at
  instance creation, and the blocks of a batch are copied to the device as
  one array;
* each segment is cut into tiles of ``block_size * elems_per_thread``
  consecutive elements (no tile crosses a segment), and a grid of
  ``resident CTAs per SM x SMs`` walks the tile list, so meshes of very
  different sizes share the GPU evenly;
* INC into Dats and Mats uses the atomic form; Global reductions are reduced
  per tile and finalised per segment in tile order by a second kernel, so a
  segment's Global does not depend on what else is in the batch.

There is no counterpart in the reference: pyop2/cuda.py launched one
par_loop at a time with a host synchronise after each (pyop2/cuda.py:656-658).
"""

import copy
import struct

import numpy as np

from . import b200, codegen
from . import configuration as cfg
from ._lib import call
from .exceptions import DeviceError

TILE_DTYPE = np.dtype([("seg", "<i4"), ("pad", "<i4"), ("first", "<i8")])

# (loop signature, block size, elements per thread, min blocks) ->
# (module, BatchLayout, has finalisation, finalisation function, CTAs per SM)
_COMPILED = {}


def build_tiles(sizes, tile):
    """Tile list of a batch: segment i of ``sizes[i]`` elements is cut into
    ceil(sizes[i] / tile) tiles starting at 0, tile, 2*tile, ...  Returns the
    tiles (TILE_DTYPE; one zero entry when there are none) and each segment's
    first tile index (len(sizes) + 1 entries, the last = number of tiles)."""
    sizes = np.asarray(sizes, dtype=np.int64)
    if (sizes < 0).any() or tile < 1:
        raise ValueError("bad segment sizes or tile")
    nt = (sizes + tile - 1) // tile
    tile_first = np.zeros(len(sizes) + 1, dtype=np.int64)
    np.cumsum(nt, out=tile_first[1:])
    ntiles = int(tile_first[-1])
    tiles = np.zeros(max(ntiles, 1), dtype=TILE_DTYPE)
    if ntiles:
        seg = np.repeat(np.arange(len(sizes), dtype=np.int32), nt)
        tiles["seg"][:ntiles] = seg
        tiles["first"][:ntiles] = (np.arange(ntiles, dtype=np.int64) - tile_first[seg]) * tile
    return tiles, tile_first


def _fields(info):
    """The pointer fields of a loop instance and the object behind each:
    [(field, kind, obj)]; kind 'slots' holds (Mat, row Map, column Map)."""
    f = []
    spec = info['spec']
    for k, m in enumerate(info['maps']):
        f.append(("m%d" % k, "map", m))
    for j, m in enumerate(info['mats']):
        f.append(("mv%d" % j, "mat", m))
    if spec.mat_slots:
        seen = set()
        for s in info['specs']:
            if s.kind == "mat" and s.slot not in seen:
                seen.add(s.slot)
                f.append(("ms%d" % s.slot, "slotsrel" if spec.mat_slots_rel else "slots",
                          (info['mats'][s.slot], info['maps'][s.mslot], info['maps'][s.cmslot])))
    for j, d in enumerate(info['dats']):
        f.append(("d%d" % j, "dat", d))
    for j, g in enumerate(info['gbls']):
        f.append(("g%d" % j, "gbl", g))
    return f


def _bind(fields):
    """Parameter values (device addresses) of one loop instance."""
    vals = {}
    for name, kind, o in fields:
        if kind == "map":
            vals[name] = o._to_device().ptr
        elif kind == "mat":
            j = name[2:]
            vals[name] = o._device_values().ptr
            vals["mr" + j] = o.sparsity._d_rowptr
            vals["mc" + j] = o.sparsity._d_colidx
        elif kind == "slots":
            m, rmap, cmap = o
            vals[name] = m.sparsity._slot_table(rmap, cmap).ptr
        elif kind == "slotsrel":
            m, rmap, cmap = o
            vals[name] = m.sparsity._slot_table_rel(rmap, cmap).ptr
        elif kind == "dat":
            o._to_device()
            vals[name] = o._device.ptr
            if o.soa:
                vals["ds" + name[1:]] = o.dataset.total_size
        else:
            o._to_device()
            vals[name] = o._device.ptr
    vals["err"] = b200._state['err'].ptr
    return vals


class LoopInstance(object):
    """One par_loop kept ready for batching: ``LoopInstance(kernel,
    it_space, *args)`` with the arguments ``op2.par_loop`` takes.

    :meth:`like` makes the same loop over other objects (another mesh, other
    Dats) without re-deriving the loop signature."""

    def __init__(self, kernel, it_space, *args, form="atomic", part_size=256):
        loop = b200.ParLoop(kernel, it_space, *args)
        self._loop_args = (kernel, it_space) + tuple(args)
        self.form = form
        self.plan = None
        if form == "color":
            info = b200.loop_spec(loop, owner_mode='never', inc_mode='color', min_blocks=0)
            spec = info['spec']
            if spec.mode != "plan" or any(s.kind == "gbl" and s.access != "READ"
                                          for s in info['specs']):
                raise NotImplementedError("the coloured batched form runs indirect loops "
                                          "without Global reductions (kernel %s)" % kernel.name)
            if b200._slots_usable(info['specs']):
                spec.mat_slots = True
                spec.mat_alias = b200.mat_alias(info['specs'], info['mats'])
            self.plan = _instance_plan(info, int(part_size))
            spec.batch_part_size = int(part_size)
        elif form == "atomic":
            info = b200.loop_spec(loop, owner_mode='never', inc_mode='atomic', min_blocks=0)
            spec = info['spec']
            if spec.mode not in ("direct", "atomic"):
                raise NotImplementedError("batched loops need direct access or atomic INC "
                                          "(kernel %s)" % kernel.name)
        else:
            raise ValueError("batched form %r (atomic or color)" % form)
        self.spec = spec
        self.key = spec.key()
        self.iterset = info['iterset']
        specs = info['specs']
        written = {id(a.data) for a, s in zip(loop.args, specs)
                   if a._is_dat and s.access != "READ"}
        self.dats = list(info['dats'])
        self.gbls = list(info['gbls'])
        self.mats = list(info['mats'])
        self.written = [d for d in self.dats if id(d) in written]
        self.reducing = [g for g, s in zip(self.gbls, [s for s in specs if s.kind == "gbl"])
                         if s.access != "READ"]
        self.fields = _fields(info)
        self._finish()

    def _finish(self):
        self.size = int(self.iterset.size)
        self.vals = _bind(self.fields)
        if self.plan is not None:
            d = self.plan.dptr
            self.vals.update(blkmap=d["blkmap"], offset=d["offset"], nelems=d["nelems"],
                             nthrcol=d["nthrcol"], thrcol=d["thrcol"], ind_map=d["ind_map"],
                             ind_sizes=d["ind_sizes"], ind_offs=d["ind_offs"],
                             loc_map=d["loc_map"])
        self.params = codegen.ParamLayout(self.spec).pack(self.size, 0, self.size, self.vals)

    def recast(self, form, part_size=256):
        """The same loop over the same objects in another batched form."""
        return LoopInstance(*self._loop_args, form=form, part_size=part_size)

    def like(self, subs):
        """The same loop with objects replaced: ``subs`` maps each object of
        this instance (iteration Set, Maps, Dats, Mats, Globals) to its
        replacement; objects not listed are shared.  Replacements must have
        the types, dims and arities of the originals (atomic form only: a
        coloured instance's plan belongs to its own Maps)."""
        if self.plan is not None:
            raise NotImplementedError("like() of a coloured batched instance")
        new = object.__new__(LoopInstance)
        new.form, new.plan = self.form, None
        new._loop_args = None
        new.spec, new.key = self.spec, self.key
        by_id = {id(k): v for k, v in subs.items()}   # Maps compare by structure
        r = lambda o: by_id.get(id(o), o)  # noqa: E731
        new.iterset = r(self.iterset)
        new.dats = [r(d) for d in self.dats]
        new.gbls = [r(g) for g in self.gbls]
        new.mats = [r(m) for m in self.mats]
        new.written = [r(d) for d in self.written]
        new.reducing = [r(g) for g in self.reducing]
        new.fields = [(n, k, tuple(r(x) for x in o) if k in ("slots", "slotsrel") else r(o))
                      for n, k, o in self.fields]
        for (n, k, o), (_, _, o2) in zip(self.fields, new.fields):
            if k in ("dat", "gbl") and (o.dtype != o2.dtype or o.cdim != o2.cdim):
                raise ValueError("replacement for %s differs in type or dim" % n)
            if k == "map" and o.dim != o2.dim:
                raise ValueError("replacement for %s differs in arity" % n)
        new._finish()
        return new

    def patch(self, ptrs):
        if self.plan is not None:
            raise NotImplementedError("patch() of a coloured batched instance")
        return self._patch(ptrs)

    def _patch(self, ptrs):
        """A :class:`PatchedInstance` of this loop whose arguments bound to
        the objects in ``ptrs`` (object -> device address) read and write the
        given addresses instead: raw device memory of the same layout (e.g.
        a request's arena).  Maps, Sparsity and sizes are shared."""
        layout = codegen.ParamLayout(self.spec)
        buf = bytearray(self.params)
        by_id = {id(k): v for k, v in ptrs.items()}
        hit = 0
        for name, kind, o in self.fields:
            if kind in ("dat", "gbl", "mat") and id(o) in by_id:
                struct.pack_into("<Q", buf, layout.offset(name), int(by_id[id(o)]))
                hit += 1
        if hit == 0:
            raise ValueError("none of the objects to patch is an argument of the loop")
        return PatchedInstance(self, bytes(buf))

    def sync(self):
        """Upload Dats and Globals whose host copy is newer."""
        for d in self.dats:
            if d._state is b200.HOST:
                d._to_device()
        for g in self.gbls:
            if g._state is b200.HOST:
                g._to_device()

    def mark(self):
        """Record that the device copies of written data are now newer."""
        for d in self.written:
            d._state = b200.DEVICE
            d._wgen += 1
        for g in self.reducing:
            g._state = b200.DEVICE
        for m in self.mats:
            m._state = b200.DEVICE
            m._is_zero = False


class PatchedInstance(object):
    """A loop instance made by :meth:`LoopInstance.patch`: the template's
    signature with its own parameter block.  Its data lives in raw device
    memory owned by the caller, so there is no host copy to synchronise."""

    __slots__ = ("spec", "key", "size", "params")
    form = "atomic"     # patched instances run the atomic batched form
    plan = None

    def __init__(self, template, params):
        self.spec, self.key, self.size = template.spec, template.key, template.size
        self.params = params

    def sync(self):
        pass

    def mark(self):
        pass


class BatchLoop(object):
    """All ``instances`` (LoopInstance, one signature) in one launch.

    ``block_size`` threads per CTA, ``elems_per_thread`` elements per thread
    per tile, ``min_blocks`` the stub's __launch_bounds__ minimum CTAs per SM
    (0: none), ``ctas_per_sm`` caps the persistent grid (0: all resident)."""

    def __init__(self, instances, block_size=None, elems_per_thread=1, min_blocks=0,
                 ctas_per_sm=0):
        if not instances:
            raise ValueError("a batch needs at least one instance")
        self.instances = list(instances)
        key = self.instances[0].key
        for n, inst in enumerate(self.instances):
            if inst.key != key:
                raise ValueError("instance %d of the batch has a different loop signature" % n)
        spec = copy.copy(self.instances[0].spec)
        spec.block_size = int(block_size or cfg.cfg['block_size'])
        spec.batch = int(elems_per_thread)
        spec.min_blocks = int(min_blocks)
        if spec.batch < 1:
            raise ValueError("elems_per_thread must be >= 1")
        self.spec = spec
        self.form = self.instances[0].form
        self.config = dict(block_size=spec.block_size, elems_per_thread=spec.batch,
                           min_blocks=spec.min_blocks, ctas_per_sm=int(ctas_per_sm))
        if self.form == "color":
            self.config = dict(form="color", part_size=spec.batch_part_size,
                               block_size=spec.block_size, min_blocks=spec.min_blocks,
                               ctas_per_sm=int(ctas_per_sm))
        self.smem = max((i.plan.nshared for i in self.instances if i.plan is not None), default=0)
        ckey = (key, spec.block_size, spec.batch, spec.min_blocks)
        hit = _COMPILED.get(ckey)
        if hit is None:
            module = b200._get_module(spec)
            layout = codegen.BatchLayout(spec)
            has_fin = len(layout.fields) > 5
            fin = module.function(codegen.batch_stub_names(spec)[1]) if has_fin else 0
            hit = _COMPILED[ckey] = (module, layout, has_fin, fin)
        self.module, self.layout, self.has_fin, self.fin = hit
        if self.smem > b200._state['smem_optin']:
            raise DeviceError("coloured batch needs %d bytes of shared memory per block" % self.smem)
        self.module.ensure_smem(self.smem)
        occ = self.module.occupancy(self.module.fn, spec.block_size, self.smem)
        if self.form == "color":
            self._init_colored(occ, int(ctas_per_sm))
            return
        # segments and tiles
        sizes = np.array([inst.size for inst in self.instances], dtype=np.int64)
        tiles, tile_first = build_tiles(sizes, spec.block_size * spec.batch)
        ntiles = int(tile_first[-1])
        self.ntiles, self.nsegs = ntiles, len(sizes)
        self.elements = int(sizes.sum())
        # one upload: parameter blocks | tiles | first tile per segment
        segs = b"".join(i.params for i in self.instances)
        o_tiles = (len(segs) + 15) // 16 * 16
        o_first = o_tiles + tiles.nbytes
        host = np.zeros(o_first + tile_first.nbytes, dtype=np.uint8)
        host[:len(segs)] = np.frombuffer(segs, dtype=np.uint8)
        host[o_tiles:o_first] = tiles.view(np.uint8)
        host[o_first:] = tile_first.view(np.uint8)
        self._meta = b200._upload(host)
        base = self._meta.ptr
        vals = dict(segs=base, tiles=base + o_tiles, tile_first=base + o_first,
                    ntiles=ntiles, nsegs=self.nsegs)
        self._gpart = []
        for name in self.layout.fields[5:]:
            ctype, cdim, _ = spec.gbls[int(name[5:])]
            item = np.dtype(_CTYPES[ctype]).itemsize
            buf = b200.DeviceBuffer(max(ntiles, 1) * cdim * item)
            self._gpart.append(buf)
            vals[name] = buf.ptr
        self._params = self.layout.pack(vals)
        if occ < 1:
            raise DeviceError("batched stub %s cannot be resident at block size %d"
                              % (spec.kernel_name, spec.block_size))
        if ctas_per_sm:
            occ = min(occ, int(ctas_per_sm))
        self.grid = int(min(ntiles, occ * b200._state['sm_count']))
        self.fin_grid = (self.nsegs * 32 + 255) // 256
        self.consts = b200.base.Const._definitions()

    def _init_colored(self, occ, ctas_per_sm):
        """Tiles of the coloured form: for colour c, every segment's blocks
        of colour c (positions in its blkmap); one launch per colour."""
        spec = self.spec
        sizes = np.array([inst.size for inst in self.instances], dtype=np.int64)
        self.nsegs = len(sizes)
        self.elements = int(sizes.sum())
        ncol = max((i.plan.ncolors for i in self.instances), default=0)
        per = []
        for c in range(ncol):
            segs, firsts = [], []
            for s, inst in enumerate(self.instances):
                pl = inst.plan
                if c >= pl.ncolors:
                    continue
                ncb = list(pl.ncolblk_host)[:pl.ncolors]
                c0 = sum(ncb[:c])
                segs += [s] * ncb[c]
                firsts += list(range(c0, c0 + ncb[c]))
            t = np.zeros(max(len(segs), 1), dtype=TILE_DTYPE)
            if segs:
                t["seg"][:len(segs)] = segs
                t["first"][:len(segs)] = firsts
            per.append((t, len(segs)))
        segs_b = b"".join(i.params for i in self.instances)
        o_tiles = (len(segs_b) + 15) // 16 * 16
        total = o_tiles + sum(t.nbytes for t, _ in per)
        host = np.zeros(max(total, 16), dtype=np.uint8)
        host[:len(segs_b)] = np.frombuffer(segs_b, dtype=np.uint8)
        offs, o = [], o_tiles
        for t, _ in per:
            host[o:o + t.nbytes] = t.view(np.uint8)
            offs.append(o)
            o += t.nbytes
        self._meta = b200._upload(host)
        base = self._meta.ptr
        if occ < 1:
            raise DeviceError("batched stub %s cannot be resident at block size %d"
                              % (spec.kernel_name, spec.block_size))
        if ctas_per_sm:
            occ = min(occ, ctas_per_sm)
        self._gpart = []
        self._colour_launches = []
        for (t, n), off in zip(per, offs):
            if n == 0:
                continue
            params = self.layout.pack(dict(segs=base, tiles=base + off, tile_first=0, ntiles=n,
                                           nsegs=self.nsegs))
            self._colour_launches.append((int(min(n, occ * b200._state['sm_count'])), params))
        self.ntiles = sum(n for _, n in per)
        self.grid = max((g for g, _ in self._colour_launches), default=0)
        self.consts = b200.base.Const._definitions()

    @property
    def launches(self):
        """Kernels one :meth:`launch` issues."""
        if self.form == "color":
            return len(self._colour_launches)
        return (1 if self.grid else 0) + (1 if self.has_fin and self.nsegs else 0)

    def launch(self, sync_host=True):
        """Run every instance (asynchronous on the op2 stream).  With
        ``sync_host`` first upload data whose host copy is newer, and mark
        written data as newer on the device afterwards."""
        if sync_host:
            for inst in self.instances:
                inst.sync()
        b200._sync_consts(self.module, self.consts)
        if self.form == "color":
            for grid, params in self._colour_launches:
                call("op2b_launch", self.module.fn, grid, self.spec.block_size, self.smem, 0,
                     params, self.layout.nbytes)
        elif self.grid:
            call("op2b_launch", self.module.fn, self.grid, self.spec.block_size, 0, 0,
                 self._params, self.layout.nbytes)
        if self.has_fin and self.nsegs:
            call("op2b_launch", self.fin, self.fin_grid, 256, 0, 0, self._params, self.layout.nbytes)
        if sync_host:
            for inst in self.instances:
                inst.mark()


_PLANS = {}


def _instance_plan(info, part_size):
    """The GPU plan (block partition, block and thread colours, INC staging)
    of a coloured batched instance, cached per (Maps, partition size)."""
    maps, dats, stages, races = info['maps'], info['dats'], info['stages'], info['races']
    iterset = info['iterset']
    key = (iterset.size, part_size, tuple((id(maps[st[1]]), tuple(st[4])) for st in stages),
           tuple((tuple((id(m), ix) for m, ix in ents), size) for ents, size in races))
    hit = _PLANS.get(key)
    if hit is not None and all(r() is not None for r in hit[1]):
        return hit[0]
    import weakref
    plan = b200.DevicePlan(iterset.size, part_size,
                           [(maps[st[1]], st[4], np.dtype(dats[st[0]].dtype).itemsize * st[3])
                            for st in stages],
                           [(ents, size) for ents, size in races], staging=True,
                           thread_coloring=True)
    plan._keep = list(maps)
    _PLANS[key] = (plan, [weakref.ref(m) for m in maps])
    return plan


_CTYPES = {"double": np.float64, "float": np.float32, "int": np.int32, "unsigned int": np.uint32,
           "long long": np.int64, "unsigned long long": np.uint64, "long": np.int64,
           "unsigned long": np.uint64, "short": np.int16, "char": np.int8}
