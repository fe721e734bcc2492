"""CUDA source generation for par_loop stubs (compiled by NVRTC for sm_100a).

One stub is generated per loop signature.  Its single parameter is a struct
(``op2b_params``) of 8-byte fields, packed by the host (:class:`ParamLayout`).

Direct loops (no Map, no Mat) run a grid-stride loop, one thread per element.
Indirect loops run one CTA per plan block of the current block colour; the
host launches the colours in order (pyop2/cuda.py:757-800 did the same with a
synchronise per colour).  Per element the stub:

* loads READ / RW / INC(direct) rows into registers with vector loads and
  gathers READ rows through the Map (pyop2/host.py:91-134 gave the kernel
  pointers into the global arrays; the kernel now sees register copies);
* passes WRITE / RW indirect rows and direct WRITE rows as global pointers;
* gives INC indirect args zeroed register rows, and after the kernel adds them
  into shared memory at the plan's block-local slot (``loc_map``), one thread
  colour at a time, then adds each shared row once into the Dat
  (cuda_indirect_loop.jinja2:105-210 did this with a staged gather of every
  indirect Dat);
* for a Mat arg builds the local tensor the sequential wrapper builds
  (pyop2/sequential.py:62-70, host.py:145-207) and adds it into the CSR values
  at the positions found by binary search in the row, in the thread-colour
  section (the plan colours the Mat's row Map), so no atomics are needed;
* keeps Global reductions in registers and reduces them deterministically on
  the device (op2b_device.cuh: op2b_reduce).
"""

import os
import re
import struct

_DEVICE_HEADER = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "device",
                              "op2b_device.cuh")

_ACC_CODE = {"READ": 0, "WRITE": 1, "RW": 2, "INC": 3, "MIN": 4, "MAX": 5}
_RED_OP = {"INC": 0, "MIN": 1, "MAX": 2}


def device_header():
    with open(_DEVICE_HEADER) as f:
        return f.read()


class ArgSpec(object):
    """Static description of one actual par_loop argument.

    kind: 'gbl' | 'direct' | 'ind' | 'vec' | 'its' | 'mat'
    slot: unique Dat / Global / Mat slot;  mslot: unique Map slot (rmap for a Mat)
    cmslot: column Map slot of a Mat;  idx: Map index ('ind') or iteration
    space index ('its');  arity / carity: Map arities;  ext: extent of the
    iteration index;  rm, cm: Mat block dims;  soa: SoA Dat;
    loc_rows: plan loc_map rows of an INC arg (one per unwound Map index);
    stage: plan staging pair of an INC arg."""

    __slots__ = ("kind", "access", "ctype", "cdim", "slot", "mslot", "cmslot", "idx", "cidx",
                 "arity", "carity", "ext", "cext", "rm", "cm", "soa", "loc_rows", "stage",
                 "ro")

    def __init__(self, **kw):
        for k in self.__slots__:
            setattr(self, k, kw.get(k))

    def key(self):
        return tuple(tuple(v) if isinstance(v, list) else v
                     for v in (getattr(self, k) for k in self.__slots__))


class LoopSpec(object):
    """Everything the generator needs about one loop."""

    def __init__(self, kernel_name, kernel_code, extents, args, dats, maps, mats, gbls,
                 consts, indirect, stages, block_size, fmad, min_blocks=0, mode=None):
        self.min_blocks = int(min_blocks)
        # 'direct': no Map; 'plan': coloured blocks of a GPU plan; 'atomic':
        # one grid-stride launch, INC args added with atomics
        self.mode = mode or ("plan" if indirect else "direct")
        self.owner = None   # owner-computes description (mode 'owner')
        # elements per thread of a batched launch (0: not batched); see _batch_body
        self.batch = 0
        # scalar Mats found through scatter-slot tables (op2b_mat_slots_build)
        # instead of a row search per entry (atomic and batched forms)
        self.mat_slots = False
        # Mat slot whose scatter-slot table each Mat slot reads (Mats on one
        # Sparsity through the same Map pair share one table and one load)
        self.mat_alias = ()
        # scalar Mat entries added right after the kernel call of their
        # (i0, i1) instead of after the whole local tensor (atomic form with
        # slot tables): one entry live at a time instead of the whole tensor
        self.mat_per_entry = False
        # per-entry adds read the compact in-row table (op2b_mat_slots_rel_build)
        self.mat_slots_rel = False
        # (row blocks, column blocks) of a 2-d iteration space handed to
        # different warps of the atomic form (each warp evaluates its block
        # of local positions for 32 elements); None: one thread per element
        self.itspace_split = None
        # elements per thread per round of a direct stub (their loads issued
        # together before the kernel calls)
        self.direct_unroll = 1
        # (Dat slot, Map slot) pairs of the atomic form read from a gathered
        # copy: row k of element e at (e * arity + k), no Map read
        self.gathered = ()
        # staged form over a locality partition (mode 'staged'): map_stage
        # {map slot: staged Map}, stage_arity, row_base (first loc row of each
        # staged Map), read_pairs / inc_pairs [(Dat slot, staged Map, ctype,
        # cdim)] staged / accumulated in shared memory
        self.region = None
        self.kernel_name = kernel_name
        self.kernel_code = kernel_code
        self.extents = tuple(extents)
        self.args = args              # [ArgSpec]
        self.dats = dats              # [(ctype, soa)] per unique Dat slot
        self.maps = maps              # [arity] per unique Map slot
        self.mats = mats              # [ctype] per Mat slot
        self.gbls = gbls              # [(ctype, cdim, access)] per Global slot
        self.consts = consts          # [(name, ctype, cdim)]
        self.indirect = indirect
        self.stages = stages          # [(dat slot, map slot, ctype, cdim, [idx...])] INC pairs
        self.block_size = block_size
        self.fmad = fmad

    def key(self):
        return (self.kernel_name, self.kernel_code, self.extents,
                tuple(a.key() for a in self.args), tuple(self.dats), tuple(self.maps),
                tuple(self.mats), tuple(self.gbls), tuple(self.consts), self.indirect,
                tuple((s[0], s[1], s[2], s[3], tuple(s[4])) for s in self.stages),
                self.block_size, self.fmad, self.min_blocks, self.mode,
                tuple(sorted(self.owner.items())) if self.owner else None, self.batch,
                self.mat_slots, _freeze(self.region), tuple(self.mat_alias),
                self.mat_per_entry, self.itspace_split, self.direct_unroll,
                self.mat_slots_rel, tuple(self.gathered))

    @property
    def needs_coloring(self):
        return any(a.kind == "mat" or (a.kind in ("ind", "vec", "its") and a.access == "INC")
                   for a in self.args)


def _freeze(v):
    if isinstance(v, dict):
        return tuple(sorted((k, _freeze(x)) for k, x in v.items()))
    if isinstance(v, (list, tuple)):
        return tuple(_freeze(x) for x in v)
    return v


class ParamLayout(object):
    """Field order of op2b_params.  The header is (set_size i64, col_first i32,
    col_n i32, start i64, end i64); every other field is 8 bytes."""

    HEADER = "<qiiqq"
    COL_OFFSET = 8

    def __init__(self, spec):
        f = []
        if spec.mode == "owner":
            f += ["inc_ptr", "inc_list"]
        if spec.mode == "gather":
            f += ["inc_ptr", "inc_list", "inc_order"]
        if spec.mode == "plan":
            f += ["blkmap", "offset", "nelems", "nthrcol", "thrcol", "ind_map", "ind_sizes",
                  "ind_offs", "loc_map"]
        if spec.mode == "staged":
            f += ["rg_order", "rg_boff", "rg_tlist", "rg_toff", "rg_tcnt", "rg_loc", "rg_thrcol",
                  "rg_nthrcol"]
        for j in range(len(spec.dats)):
            f.append("d%d" % j)
            if spec.dats[j][1]:
                f.append("ds%d" % j)
        for k in range(len(spec.maps)):
            f.append("m%d" % k)
        for j in range(len(spec.mats)):
            f += ["mv%d" % j, "mr%d" % j, "mc%d" % j]
            if spec.mat_slots:
                f.append("ms%d" % j)
            if spec.mode == "lma":
                f.append("lm%d" % j)
        if spec.mode == "lma":
            f += ["ld%d" % k for k in range(len(spec.stages))]
        for j, g in enumerate(spec.gbls):
            f.append("g%d" % j)
            if g[2] != "READ":
                f += ["gp%d" % j, "gc%d" % j]
            if gbl_init_fields(g):
                f += ["gf%d" % j] + ["gv%d_%d" % (j, k) for k in range(g[1])]
        f.append("err")
        self.fields = f
        self.index = {n: i for i, n in enumerate(f)}
        self.fmt = self.HEADER + "Q" * len(f)
        self.nbytes = struct.calcsize(self.fmt)

    def pack(self, set_size, start, end, values):
        return struct.pack(self.fmt, set_size, 0, 0, start, end,
                           *[int(values.get(n, 0)) for n in self.fields])

    def offset(self, name):
        """Byte offset of a field in the packed block."""
        return struct.calcsize(self.HEADER) + 8 * self.index[name]


def _struct_decl(spec, layout):
    lines = ["struct op2b_params {", "  op2b_i64 set_size;", "  int col_first, col_n;",
             "  op2b_i64 start, end;"]
    types = {"blkmap": "const int *", "offset": "const int *", "nelems": "const int *",
             "nthrcol": "const int *", "thrcol": "const int *", "ind_map": "const int *",
             "ind_sizes": "const int *", "ind_offs": "const int *", "loc_map": "const short *",
             "err": "int *", "inc_ptr": "const int *", "inc_list": "const int *",
             "inc_order": "const int *",
             "rg_order": "const int *", "rg_boff": "const int *", "rg_tlist": "const int *",
             "rg_toff": "const int *", "rg_tcnt": "const int *", "rg_loc": "const short *",
             "rg_thrcol": "const int *", "rg_nthrcol": "const int *"}
    for n in layout.fields:
        if n in types:
            t = types[n]
        elif n.startswith("ds"):
            t = "op2b_i64 "
        elif n.startswith("d"):
            t = "%s *" % spec.dats[int(n[1:])][0]
        elif n.startswith("mv"):
            t = "%s *" % spec.mats[int(n[2:])]
        elif n.startswith("lm"):
            t = "%s *" % spec.mats[int(n[2:])]
        elif n.startswith("ld"):
            t = "%s *" % spec.stages[int(n[2:])][2]
        elif n.startswith("mr") or n.startswith("mc") or n.startswith("m"):
            t = "const int *"
        elif n.startswith("gf"):
            t = "op2b_i64 "
        elif n.startswith("gv"):
            t = "op2b_u64 "
        elif n.startswith("gp"):
            t = "%s *" % spec.gbls[int(n[2:])][0]
        elif n.startswith("gc"):
            t = "unsigned *"
        elif n.startswith("g"):
            t = "%s *" % spec.gbls[int(n[1:])][0]
        else:
            raise AssertionError(n)
        lines.append("  %s%s;" % (t, n))
    lines.append("};")
    return "\n".join(lines)


def _bounds(spec):
    if spec.min_blocks:
        return "__launch_bounds__(%d, %d)" % (spec.block_size, spec.min_blocks)
    return "__launch_bounds__(%d)" % spec.block_size


def stub_name(spec):
    """Symbol of the stub: op2b_<user kernel name> (distinct per loop in
    profiles)."""
    import re
    return "op2b_" + re.sub(r"[^A-Za-z0-9_]", "_", spec.kernel_name)


def _mark_inline(code, name):
    import re
    pat = re.compile(r"(^|[;}\s])((?:static\s+|inline\s+)*void\s+%s\s*\()" % re.escape(name))
    m = pat.search(code)
    if not m:
        return code
    return code[:m.start(2)] + "__forceinline__ " + code[m.start(2):]


def generate(spec):
    """Return (source, ParamLayout, stub name) for a LoopSpec."""
    layout = ParamLayout(spec)
    out = []
    w = out.append
    w(device_header())
    for name, ctype, cdim in spec.consts:
        if cdim == 1:
            w("__constant__ %s %s;" % (ctype, name))
        else:
            w("__constant__ %s %s[%d];" % (ctype, name, cdim))
    w(_struct_decl(spec, layout))
    w("#define OP2_STRIDE(a, idx) (a)[idx]")
    # the user's code lives in its own namespace, so no local name of a stub
    # can hide the kernel (the reference's tests call many kernels "k")
    w("namespace op2b_user {")
    w(_mark_inline(spec.kernel_code, spec.kernel_name))
    w("}  // namespace op2b_user")
    w("#undef OP2_STRIDE")
    if spec.batch:
        w(_enter(_batch_plan_body(spec) if spec.mode == "plan" else _batch_body(spec)))
        return "\n".join(out), layout, batch_stub_names(spec)[0]
    body = {"plan": _indirect_body, "atomic": _atomic_body, "lma": _atomic_body,
            "direct": _direct_body, "owner": _owner_body, "staged": _staged_body,
            "gather": _gather_body}[spec.mode](spec)
    w(_enter(body))
    return "\n".join(out), layout, stub_name(spec)


def _enter(body):
    """Every kernel of a stub begins with op2b_stub_enter() (wait for the
    previous kernel on the stream, let the next one be scheduled)."""
    out = []
    for line in body.split("\n"):
        out.append(line)
        if line.startswith('extern "C" __global__') and line.rstrip().endswith("{"):
            out.append("  op2b_stub_enter();")
    return "\n".join(out)


# ------------------------------------------------------------------ helpers
def _ro(a):
    return "true" if a.ro else "false"


# A reduction Global's value before the loop may travel in the launch
# parameters (fields gf<slot>: flag, gv<slot>_<k>: component k's bits in an
# 8-byte word) instead of its device copy, for these types and at most
# GBL_INIT_MAX components: a Global the host has just created or set then
# needs no upload.  Expressions turning the word back into the value:
_GBL_INIT = {"double": "__longlong_as_double((long long)%s)",
             "float": "__int_as_float((int)(unsigned)%s)",
             "int": "(int)%s", "unsigned int": "(unsigned int)%s",
             "long long": "(long long)%s", "unsigned long long": "(unsigned long long)%s"}
GBL_INIT_MAX = 4


def gbl_init_fields(g):
    """Whether a Global slot (ctype, cdim, access) carries its value before
    the loop in the launch parameters."""
    return g[2] != "READ" and g[0] in _GBL_INIT and g[1] <= GBL_INIT_MAX


def _gbl_init(a, k):
    return _GBL_INIT[a.ctype] % ("p.gv%d_%d" % (a.slot, k))


def _gbl_prologue(spec, lines):
    for n, a in enumerate(spec.args):
        if a.kind != "gbl":
            continue
        t, c = a.ctype, a.cdim
        if a.access == "READ":
            lines.append("  %s g%d_l[%d];" % (t, n, c))
            lines.append("  for (int k = 0; k < %d; ++k) g%d_l[k] = p.g%d[k];" % (c, n, a.slot))
        else:
            lines.append("  %s r%d[%d];" % (t, n, c))
            if a.access == "INC":
                lines.append("  op2b_zero(r%d);" % n)
            elif gbl_init_fields(spec.gbls[a.slot]):
                for k in range(c):
                    lines.append("  r%d[%d] = p.gf%d ? %s : p.g%d[%d];"
                                 % (n, k, a.slot, _gbl_init(a, k), a.slot, k))
            else:
                lines.append("  for (int k = 0; k < %d; ++k) r%d[k] = p.g%d[k];" % (c, n, a.slot))


def _gbl_epilogue(spec, lines):
    for n, a in enumerate(spec.args):
        if a.kind == "gbl" and a.access != "READ":
            if gbl_init_fields(spec.gbls[a.slot]):
                lines.append("  { const %s i%d[%d] = {%s};" % (
                    a.ctype, n, a.cdim, ", ".join(_gbl_init(a, k) for k in range(a.cdim))))
                lines.append("    op2b_reduce<%d, %s, %d>(r%d, p.g%d, p.gp%d, p.gc%d, p.gf%d != 0, i%d); }"
                             % (_RED_OP[a.access], a.ctype, a.cdim, n, a.slot, a.slot, a.slot,
                                a.slot, n))
            else:
                lines.append("  op2b_reduce<%d, %s, %d>(r%d, p.g%d, p.gp%d, p.gc%d);" %
                             (_RED_OP[a.access], a.ctype, a.cdim, n, a.slot, a.slot, a.slot))


def _direct_row(a, n, e, lines_pre, lines_post, indent):
    """Code for a direct Dat arg of element e; returns the kernel argument."""
    t, c, j = a.ctype, a.cdim, a.slot
    if a.soa:
        lines_pre.append("%s__align__(16) %s a%d[%d];" % (indent, t, n, c))
        if a.access != "WRITE" or True:
            lines_pre.append("%sop2b_load_soa(a%d, p.d%d, %s, p.ds%d);" % (indent, n, j, e, j))
        if a.access != "READ":
            lines_post.append("%sop2b_store_soa(p.d%d, %s, p.ds%d, a%d);" % (indent, j, e, j, n))
        return "a%d" % n
    if a.access == "WRITE":
        # The whole row is written back from registers with vector stores (as
        # the reference CUDA backend's staged direct args, which wrote back the
        # full row, cuda_direct_loop.jinja2:63-65); components the kernel does
        # not write become 0.
        lines_pre.append("%s__align__(16) %s a%d[%d]; op2b_zero(a%d);" % (indent, t, n, c, n))
        lines_post.append("%sop2b_store(p.d%d + (op2b_i64)(%s) * %d, a%d);" % (indent, j, e, c, n))
        return "a%d" % n
    lines_pre.append("%s__align__(16) %s a%d[%d];" % (indent, t, n, c))
    lines_pre.append("%sop2b_load<%s, %d, %s>(a%d, p.d%d + (op2b_i64)(%s) * %d);" %
                     (indent, t, c, _ro(a), n, j, e, c))
    if a.access != "READ":
        lines_post.append("%sop2b_store(p.d%d + (op2b_i64)(%s) * %d, a%d);" % (indent, j, e, c, n))
    return "a%d" % n


def _kernel_call(spec, argexprs, indent):
    itargs = ["i%d" % k for k in range(len(spec.extents))]
    return "%sop2b_user::%s(%s);" % (indent, spec.kernel_name, ", ".join(argexprs + itargs))


def _direct_element_parts(spec, ind, e, sfx):
    """(row declarations and loads, kernel call, stores) of element ``e``
    of a direct loop, its row variables suffixed ``sfx``."""
    pre, post, exprs = [], [], []
    for n, a in enumerate(spec.args):
        if a.kind == "gbl":
            exprs.append("g%d_l" % n if a.access == "READ" else "r%d" % n)
        else:
            p0, q0 = [], []
            x = _direct_row(a, n, e, p0, q0, ind)
            ren = lambda t, n=n: re.sub(r"\ba%d\b" % n, "a%d%s" % (n, sfx), t)  # noqa: E731
            pre += [ren(t) for t in p0]
            post += [ren(t) for t in q0]
            exprs.append(ren(x))
    call = _itspace_open(spec, ind)
    call.append(_kernel_call(spec, exprs, ind + "  " * len(spec.extents)))
    call += _itspace_close(spec, ind)
    return pre, call, post


def _direct_element(spec, ind):
    """Lines computing element ``e`` of a direct loop."""
    pre, post, exprs = [], [], []
    for n, a in enumerate(spec.args):
        if a.kind == "gbl":
            exprs.append("g%d_l" % n if a.access == "READ" else "r%d" % n)
        else:
            exprs.append(_direct_row(a, n, "e", pre, post, ind))
    L = list(pre)
    L += _itspace_open(spec, ind)
    L.append(_kernel_call(spec, exprs, ind + "  " * len(spec.extents)))
    L += _itspace_close(spec, ind)
    L += post
    return L


def _direct_body(spec):
    bs = spec.block_size
    U = spec.direct_unroll
    L = ["extern \"C\" __global__ void %s %s(const op2b_params p) {" % (_bounds(spec), stub_name(spec))]
    _gbl_prologue(spec, L)
    if U > 1:
        # U elements per thread per round, one grid stride apart: all their
        # rows are loaded before any kernel call and stored after all of
        # them, so the loads of the U elements are in flight together
        # (elements of a direct loop touch only their own rows)
        L.append("  const op2b_i64 stride = (op2b_i64)gridDim.x * %d;" % bs)
        L.append("  for (op2b_i64 e0 = p.start + (op2b_i64)blockIdx.x * %d + threadIdx.x; e0 < p.end;"
                 " e0 += stride * %d) {" % (bs, U))
        parts = []
        for u in range(U):
            L.append("    const op2b_i64 e_%d = e0 + %d * stride;" % (u, u))
            L.append("    const bool ok_%d = e_%d < p.end;" % (u, u))
            parts.append(_direct_element_parts(spec, "      ", "e_%d" % u, "_%d" % u))
        for u, (pre, call, post) in enumerate(parts):
            decls, loads = [], []
            for x in pre:
                x = x.strip()
                if x.startswith("__align__"):
                    cut = x.index(";") + 1
                    decls.append("    " + x[:cut])
                    x = x[cut:].strip()
                if x:
                    loads.append("      " + x)
            L += decls
            if loads:
                L.append("    if (ok_%d) {" % u)
                L += loads
                L.append("    }")
        for u, (pre, call, post) in enumerate(parts):
            L.append("    if (ok_%d) {" % u)
            L += call
            L.append("    }")
        for u, (pre, call, post) in enumerate(parts):
            if post:
                L.append("    if (ok_%d) {" % u)
                L += post
                L.append("    }")
        L.append("  }")
        _gbl_epilogue(spec, L)
        L.append("}")
        return "\n".join(L)
    L.append("  for (op2b_i64 e = p.start + (op2b_i64)blockIdx.x * %d + threadIdx.x; e < p.end;"
             " e += (op2b_i64)gridDim.x * %d) {" % (bs, bs))
    L += _direct_element(spec, "    ")
    L.append("  }")
    _gbl_epilogue(spec, L)
    L.append("}")
    return "\n".join(L)


def _itspace_open(spec, indent, ranges=None):
    out = []
    for k, ext in enumerate(spec.extents):
        lo, hi = ranges[k] if ranges else (0, ext)
        out.append("%s#pragma unroll" % (indent + "  " * k))
        out.append("%sfor (int i%d = %d; i%d < %d; ++i%d) {" % (indent + "  " * k, k, lo, k, hi, k))
    return out


def _split_ranges(spec):
    """The local-position blocks of an itspace split: [((r0, r1), (c0, c1))]."""
    (nr, nc), (e0, e1) = spec.itspace_split, spec.extents
    rb = [(e0 * i // nr, e0 * (i + 1) // nr) for i in range(nr)]
    cb = [(e1 * j // nc, e1 * (j + 1) // nc) for j in range(nc)]
    return [(r, c) for r in rb for c in cb]


def _itspace_close(spec, indent):
    return ["%s}" % (indent + "  " * k) for k in range(len(spec.extents) - 1, -1, -1)]


def _indirect_body(spec):
    L = ["extern \"C\" __global__ void %s %s(const op2b_params p) {" % (_bounds(spec), stub_name(spec))]
    L.append("  if ((int)blockIdx.x >= p.col_n) return;")
    L.append("  const int blk = p.blkmap[p.col_first + blockIdx.x];")
    L += _plan_block(spec)
    L.append("}")
    return "\n".join(L)


def _plan_block(spec, batched=False):
    """Lines running block ``blk`` of a plan (coloured form): the body of
    the reference's indirect-loop template (cuda_indirect_loop.jinja2)
    restated -- INC rows staged in shared memory at the plan's loc_map slots,
    thread colours serialising the shared adds and the Mat adds, the block's
    rows added to the Dats once at the end (block colours keep concurrently
    running blocks apart).  ``batched``: the block is one tile of a batched
    coloured launch (no Global reductions; a barrier before the block reuses
    shared memory)."""
    bs = spec.block_size
    ninds = len(spec.stages)
    coloured = spec.needs_coloring
    L = []
    if batched:
        L.append("  __syncthreads();")
    L.append("  const int start = p.offset[blk];")
    L.append("  const int nelem = p.nelems[blk];")
    L.append("  const op2b_i64 set_size = p.set_size;")
    if ninds:
        if not batched:
            L.append("  extern __shared__ __align__(16) unsigned char op2b_smem[];")
        L.append("  int smem_off = 0;")
        nidx_prefix = 0
        for s, (dslot, mslot, t, c, idxs) in enumerate(spec.stages):
            L.append("  const int n_s%d = p.ind_sizes[blk * %d + %d];" % (s, ninds, s))
            L.append("  %s *inc_s%d = (%s *)(op2b_smem + smem_off);" % (t, s, t))
            L.append("  smem_off += (n_s%d * %d * (int)sizeof(%s) + 15) & ~15;" % (s, c, t))
            L.append("  const int *ind_s%d = p.ind_map + (op2b_i64)%d * set_size + p.ind_offs[blk * %d + %d];"
                     % (s, nidx_prefix, ninds, s))
            L.append("  for (int t = threadIdx.x; t < n_s%d * %d; t += %d) inc_s%d[t] = (%s)0;"
                     % (s, c, bs, s, t))
            nidx_prefix += len(idxs)
        L.append("  __syncthreads();")
    if not batched:
        _gbl_prologue(spec, L)
    if coloured:
        L.append("  const int ncol = p.nthrcol[blk];")
    L.append("  for (int base = 0; base < nelem; base += %d) {" % bs)
    L.append("    const int idx = base + threadIdx.x;")
    L.append("    const bool active = idx < nelem;")
    L.append("    const int e = start + idx;")
    ind = "    "
    # map rows (needed by the kernel call and by the colour section)
    used_maps = sorted({a.mslot for a in spec.args if a.kind in ("ind", "vec", "its", "mat")} |
                       {a.cmslot for a in spec.args if a.kind == "mat"})
    for k in used_maps:
        ar = spec.maps[k]
        L.append("%s__align__(16) int mr%d[%d];" % (ind, k, ar))
        L.append("%sif (active) op2b_load<int, %d, true>(mr%d, p.m%d + (op2b_i64)e * %d);"
                 " else { for (int q = 0; q < %d; ++q) mr%d[q] = 0; }" % (ind, ar, k, k, ar, ar, k))
    # INC locals and Mat local tensors live across the colour section
    decl, pre, post, exprs = [], [], [], []
    for n, a in enumerate(spec.args):
        t, c = a.ctype, a.cdim
        if a.kind == "gbl":
            exprs.append("g%d_l" % n if a.access == "READ" else "r%d" % n)
        elif a.kind == "direct":
            exprs.append(_direct_row(a, n, "e", pre, post, ind + "  "))
        elif a.kind == "ind":
            row = "p.d%d + (op2b_i64)mr%d[%d] * %d" % (a.slot, a.mslot, a.idx, c)
            if a.access == "INC":
                decl.append("%s__align__(16) %s a%d[%d]; op2b_zero(a%d);" % (ind, t, n, c, n))
                exprs.append("a%d" % n)
            elif a.access == "READ":
                pre.append("%s  __align__(16) %s a%d[%d];" % (ind, t, n, c))
                pre.append("%s  op2b_load<%s, %d, %s>(a%d, %s);" % (ind, t, c, _ro(a), n, row))
                exprs.append("a%d" % n)
            else:
                exprs.append(row)
        elif a.kind in ("vec", "its"):
            cnt = a.arity if a.kind == "vec" else a.ext
            var = "i%d" % a.idx if a.kind == "its" else None
            if a.access in ("READ", "INC"):
                if a.access == "INC":
                    decl.append("%s__align__(16) %s a%d[%d][%d];" % (ind, t, n, cnt, c))
                    decl.append("%sfor (int q = 0; q < %d; ++q) op2b_zero(a%d[q]);" % (ind, cnt, n))
                else:
                    pre.append("%s  __align__(16) %s a%d[%d][%d];" % (ind, t, n, cnt, c))
                    for r in range(cnt):
                        pre.append("%s  op2b_load<%s, %d, %s>(a%d[%d], p.d%d + (op2b_i64)mr%d[%d] * %d);"
                                   % (ind, t, c, _ro(a), n, r, a.slot, a.mslot, r, c))
                if a.kind == "vec":
                    pre.append("%s  %s *a%d_v[%d] = {%s};" %
                               (ind, t, n, cnt, ", ".join("a%d[%d]" % (n, r) for r in range(cnt))))
                    exprs.append("a%d_v" % n)
                else:
                    exprs.append("a%d[%s]" % (n, var))
            else:
                if a.kind == "vec":
                    pre.append("%s  %s *a%d_v[%d] = {%s};" % (
                        ind, t, n, cnt, ", ".join("p.d%d + (op2b_i64)mr%d[%d] * %d" % (a.slot, a.mslot, r, c)
                                                   for r in range(cnt))))
                    exprs.append("a%d_v" % n)
                else:
                    exprs.append("p.d%d + (op2b_i64)mr%d[%s] * %d" % (a.slot, a.mslot, var, c))
        elif a.kind == "mat":
            e0, e1 = spec.extents[0], spec.extents[1]
            if a.rm * a.cm == 1:
                decl.append("%s%s A%d[%d][%d];" % (ind, t, n, e0, e1))
                exprs.append("(%s (*)[1])&A%d[i0][i1]" % (t, n))
            else:
                decl.append("%s%s A%d[%d][%d][%d][%d];" % (ind, t, n, e0, e1, a.rm, a.cm))
                exprs.append("A%d[i0][i1]" % n)
    L += decl
    if coloured:
        L.append("%sint col = -1;" % ind)
    L.append("%sif (active) {" % ind)
    L += pre
    L += _itspace_open(spec, ind + "  ")
    deep = ind + "  " + "  " * len(spec.extents)
    for n, a in enumerate(spec.args):
        if a.kind == "mat":
            if a.rm * a.cm == 1:
                L.append("%sA%d[i0][i1] = (%s)0;" % (deep, n, a.ctype))
            else:
                L.append("%sfor (int r = 0; r < %d; ++r) for (int c = 0; c < %d; ++c) A%d[i0][i1][r][c] = (%s)0;"
                         % (deep, a.rm, a.cm, n, a.ctype))
    L.append(_kernel_call(spec, exprs, deep))
    L += _itspace_close(spec, ind + "  ")
    L += post
    if coloured:
        L.append("%s  col = p.thrcol[e];" % ind)
    L.append("%s}" % ind)
    if coloured:
        L.append("%sfor (int c = 0; c < ncol; ++c) {" % ind)
        L.append("%s  if (col == c) {" % ind)
        cs = ind + "    "
        for n, a in enumerate(spec.args):
            if a.kind in ("ind", "vec", "its") and a.access == "INC":
                s = a.stage
                c_ = a.cdim
                if a.kind == "ind":
                    rows = [("a%d" % n, a.loc_rows[0])]
                else:
                    cnt = a.arity if a.kind == "vec" else a.ext
                    rows = [("a%d[%d]" % (n, r), a.loc_rows[r]) for r in range(cnt)]
                for var, lr in rows:
                    L.append("%s{ const int l = p.loc_map[(op2b_i64)%d * set_size + e];" % (cs, lr))
                    L.append("%s  for (int k = 0; k < %d; ++k) inc_s%d[l * %d + k] += %s[k]; }"
                             % (cs, c_, s, c_, var))
            elif a.kind == "mat":
                L += _mat_addto(spec, n, a, cs)
        L.append("%s  }" % ind)
        L.append("%s  __syncthreads();" % ind)
        L.append("%s}" % ind)
    L.append("  }")
    # add the block's INC rows into the Dats; pairs of the same Dat in turn
    if ninds:
        L.append("  __syncthreads();")
        seen_dats = set()
        for s, (dslot, mslot, t, c, idxs) in enumerate(spec.stages):
            if dslot in seen_dats:
                L.append("  __syncthreads();")
            seen_dats.add(dslot)
            L.append("  for (int t = threadIdx.x; t < n_s%d * %d; t += %d) {" % (s, c, bs))
            L.append("    const int r = t / %d, k = t - r * %d;" % (c, c))
            L.append("    p.d%d[(op2b_i64)ind_s%d[r] * %d + k] += inc_s%d[t];" % (dslot, s, c, s))
            L.append("  }")
    if not batched:
        _gbl_epilogue(spec, L)
    return L


def _atomic_body(spec):
    """Indirect loop without a plan: a grid-stride loop over all elements;
    INC args (Dats and Mats) are added into global memory with atomic
    reductions.  WRITE/RW indirect args are global pointers as in the
    coloured form (OP2 leaves their conflicts to the user)."""
    bs = spec.block_size
    L = ["extern \"C\" __global__ void %s %s(const op2b_params p) {" % (_bounds(spec), stub_name(spec))]
    if spec.itspace_split:
        # warp w evaluates block (w mod Q) of the local positions of the 32
        # elements 32 * (w div Q) + lane (the block is warp-uniform)
        blocks = _split_ranges(spec)
        Q = len(blocks)
        L.append("  const int lane = threadIdx.x & 31;")
        L.append("  const op2b_i64 nw = ((op2b_i64)gridDim.x * %d) >> 5;" % bs)
        L.append("  const op2b_i64 nwork = ((p.end - p.start + 31) >> 5) * %d;" % Q)
        L.append("  for (op2b_i64 w = ((op2b_i64)blockIdx.x * %d + threadIdx.x) >> 5; w < nwork; w += nw) {"
                 % bs)
        L.append("    const int q = (int)(w %% %d);" % Q)
        L.append("    const op2b_i64 e = p.start + (w / %d) * 32 + lane;" % Q)
        L.append("    if (e >= p.end) continue;")
        L.append("    switch (q) {")
        for k, rng in enumerate(blocks):
            L.append("    case %d: {" % k)
            L += _atomic_element(spec, "      ", ranges=rng)
            L.append("      break; }")
        L.append("    }")
        L.append("  }")
        L.append("}")
        return "\n".join(L)
    _gbl_prologue(spec, L)
    L.append("  for (op2b_i64 e = p.start + (op2b_i64)blockIdx.x * %d + threadIdx.x; e < p.end;"
             " e += (op2b_i64)gridDim.x * %d) {" % (bs, bs))
    L += _atomic_element(spec, "    ")
    L.append("  }")
    _gbl_epilogue(spec, L)
    L.append("}")
    return "\n".join(L)


def staged_capable(spec):
    """Loops the staged form runs: indirect Dat args only (no Mats), at
    least one indirect INC."""
    inc = False
    for a in spec.args:
        if a.kind == "mat":
            return False
        if a.kind in ("ind", "vec", "its") and a.access == "INC":
            inc = True
    return inc


_CSIZE = {"double": 8, "float": 4, "int": 4, "unsigned int": 4, "long": 8, "long long": 8,
          "unsigned long": 8, "unsigned long long": 8, "short": 2, "unsigned short": 2,
          "char": 1, "unsigned char": 1, "signed char": 1}


def staged_smem(spec, max_count):
    """Dynamic shared memory of a staged launch: the staged READ rows and
    the INC accumulators, each 16-byte aligned, at the largest per-block
    target counts."""
    R = spec.region
    nb = 0
    for (slot, st, ctype, cdim) in R["read_pairs"] + R["inc_pairs"]:
        nb += (max_count[st] * cdim * _CSIZE[ctype] + 15) // 16 * 16
    return nb


def staged_used(spec):
    R = spec.region
    used_maps = {a.mslot for a in spec.args if a.kind in ("ind", "vec", "its")}
    return sorted({R["map_stage"][k] for k in used_maps})


def _staged_prefetch(spec, R, used, bs, ind):
    """Every element of this thread (ept passes of bs threads): its loc
    rows, colour and element id, loaded as early as possible."""
    L = []
    for j in range(R["ept"]):
        L.append("%sconst int idx_%d = %d + threadIdx.x;" % (ind, j, j * bs))
        L.append("%sconst bool active_%d = idx_%d < nelem;" % (ind, j, j))
        L.append("%sconst op2b_i64 pos_%d = start + (active_%d ? idx_%d : 0);" % (ind, j, j, j))
        for st in used:
            ar = R["stage_arity"][st]
            L.append("%sint sl%d_%d[%d];" % (ind, st, j, ar))
            L.append("%s#pragma unroll" % ind)
            L.append("%sfor (int r = 0; r < %d; ++r) sl%d_%d[r] = active_%d ? (int)p.rg_loc[(op2b_i64)(%d + r) * "
                     "set_size + pos_%d] : 0;" % (ind, ar, st, j, j, R["row_base"][st], j))
        L.append("%sconst int col_%d = active_%d ? p.rg_thrcol[pos_%d] : -1;" % (ind, j, j, j))
        # positions are sorted by colour within the block: the pass's colours
        # run from its first position's to its last position's
        L.append("%sconst int clo_%d = %d < nelem ? p.rg_thrcol[start + %d] : 0;" % (ind, j, j * bs, j * bs))
        L.append("%sconst int chi_%d = %d < nelem ? p.rg_thrcol[start + min(nelem, %d) - 1] : -1;"
                 % (ind, j, j * bs, (j + 1) * bs))
        if any(a.kind == "direct" for a in spec.args):
            L.append("%sconst op2b_i64 e_%d = active_%d ? p.rg_order[pos_%d] : 0;" % (ind, j, j, j))
    return L


def _staged_copy_rows(R, used, bs, ind, dst, n, tl):
    """cp.async copies of the staged READ rows: one target id per row, the
    rows of every READ pair of the staged Map (dst % q: destination array of
    pair q; n % st / tl % st: count and target list of staged Map st)."""
    L = []
    for st in used:
        pairs = [(q, slot, t, c) for q, (slot, s_, t, c) in enumerate(R["read_pairs"]) if s_ == st]
        if not pairs:
            continue
        L.append("%sfor (int r = threadIdx.x; r < %s; r += %d) {" % (ind, n % st, bs))
        L.append("%s  const op2b_i64 g = %s[r];" % (ind, tl % st))
        if R.get("padded"):
            L.append("%s  if (g < 0) continue;   // padding slot" % ind)
        for q, slot, t, c in pairs:
            nb = c * _CSIZE[t]
            if nb % 4 == 0:
                L.append("%s  op2b_cp_async_srow<%d>(%s, r, p.d%d + g * %d);" % (ind, nb, dst % q, slot, c))
            else:
                L.append("%s  for (int k = 0; k < %d; ++k) %s[r * %d + k] = p.d%d[g * %d + k];"
                         % (ind, c, dst % q, c, slot, c))
        L.append("%s}" % ind)
    return L


def _staged_copy_rows_regs(R, used, bs, ind, KR):
    """Row copies of the staged READ rows with the target ids already in
    registers (tg<stage>_<k> holds the id of row threadIdx.x + k * bs)."""
    L = []
    for st in used:
        pairs = [(q, slot, t, c) for q, (slot, s_, t, c) in enumerate(R["read_pairs"]) if s_ == st]
        if not pairs:
            continue
        for k in range(KR[st]):
            pad = " && tg%d_%d >= 0" % (st, k) if R.get("padded") else ""
            L.append("%sif (threadIdx.x + %d < n_s%d%s) {" % (ind, k * bs, st, pad))
            L.append("%s  const int r = threadIdx.x + %d;" % (ind, k * bs))
            L.append("%s  const op2b_i64 g = tg%d_%d;" % (ind, st, k))
            for q, slot, t, c in pairs:
                nb = c * _CSIZE[t]
                if nb % 4 == 0:
                    L.append("%s  op2b_cp_async_srow<%d>(rd%d, r, p.d%d + g * %d);" % (ind, nb, q, slot, c))
                else:
                    L.append("%s  for (int k = 0; k < %d; ++k) rd%d[r * %d + k] = p.d%d[g * %d + k];"
                             % (ind, c, q, c, slot, c))
            L.append("%s}" % ind)
    return L


def _staged_flush_regs(R, bs, ind, KR):
    """Flush of the accumulated INC rows, one row per thread: the row read
    from shared memory with vector loads, added to its target with the id
    already in a register."""
    L = []
    for q, (slot, st, ctype, cdim) in enumerate(R["inc_pairs"]):
        for k in range(KR[st]):
            pad = " && tg%d_%d >= 0" % (st, k) if R.get("padded") else ""
            L.append("%sif (threadIdx.x + %d < n_s%d%s) {" % (ind, k * bs, st, pad))
            L.append("%s  __align__(16) %s cur[%d]; op2b_srow_load(cur, acc%d, threadIdx.x + %d);"
                     % (ind, ctype, cdim, q, k * bs))
            L.append("%s  op2b_atomic_row(p.d%d + (op2b_i64)tg%d_%d * %d, cur);" % (ind, slot, st, k, cdim))
            L.append("%s}" % ind)
    return L


def _staged_element(spec, R, ind, sfx=""):
    """(decl, pre, post, exprs, adds) of one element of a staged stub; with
    ``sfx`` its row variables (a<n>, a<n>_v, sl<stage>) and element id (e)
    carry that suffix, so several elements' code can share one scope."""
    parts = _staged_element_parts(spec, R, ind, "e" + sfx)
    if not sfx:
        return parts
    pat = re.compile(r"\b(a\d+|sl\d+)(_v)?\b")

    def ren(t):
        return pat.sub(lambda m: m.group(1) + sfx + (m.group(2) or ""), t)
    decl, pre, post, exprs, adds = parts
    return ([ren(t) for t in decl], [ren(t) for t in pre], [ren(t) for t in post],
            [ren(t) for t in exprs], [(ren(v), ren(r), q, c) for v, r, q, c in adds])


def _staged_element_parts(spec, R, ind, evar):
    read_of = {(sl, st): q for q, (sl, st, _, _) in enumerate(R["read_pairs"])}
    inc_of = {(sl, st): q for q, (sl, st, _, _) in enumerate(R["inc_pairs"])}
    decl, pre, post, exprs, adds = [], [], [], [], []
    for n, a in enumerate(spec.args):
        t, c = a.ctype, a.cdim
        if a.kind == "gbl":
            exprs.append("g%d_l" % n if a.access == "READ" else "r%d" % n)
            continue
        if a.kind == "direct":
            exprs.append(_direct_row(a, n, evar, pre, post, ind + "  "))
            continue
        st = R["map_stage"][a.mslot]
        cnt = a.arity if a.kind == "vec" else a.ext

        def row_ptr(rowexpr):
            return "p.d%d + (op2b_i64)tl_s%d[sl%d[%s]] * %d" % (a.slot, st, st, rowexpr, c)

        def staged_row(rowexpr):
            return "rd%d, sl%d[%s]" % (read_of[(a.slot, st)], st, rowexpr)
        if a.access == "READ":
            # staged rows into registers with vector shared-memory loads
            if a.kind == "ind":
                pre.append("%s  __align__(16) %s a%d[%d];" % (ind, t, n, c))
                pre.append("%s  op2b_srow_load(a%d, %s);" % (ind, n, staged_row(str(a.idx))))
                exprs.append("a%d" % n)
            else:
                pre.append("%s  __align__(16) %s a%d[%d][%d];" % (ind, t, n, cnt, c))
                for r in range(cnt):
                    pre.append("%s  op2b_srow_load(a%d[%d], %s);" % (ind, n, r, staged_row(str(r))))
                if a.kind == "vec":
                    pre.append("%s  %s *a%d_v[%d] = {%s};" %
                               (ind, t, n, cnt, ", ".join("a%d[%d]" % (n, r) for r in range(cnt))))
                    exprs.append("a%d_v" % n)
                else:
                    exprs.append("a%d[i%d]" % (n, a.idx))
            continue
        if a.access == "INC":
            q = inc_of[(a.slot, st)]
            if a.kind == "ind":
                decl.append("%s__align__(16) %s a%d[%d]; op2b_zero(a%d);" % (ind, t, n, c, n))
                exprs.append("a%d" % n)
                adds.append(("a%d" % n, "sl%d[%d]" % (st, a.idx), q, c))
            else:
                decl.append("%s__align__(16) %s a%d[%d][%d];" % (ind, t, n, cnt, c))
                decl.append("%sfor (int q = 0; q < %d; ++q) op2b_zero(a%d[q]);" % (ind, cnt, n))
                for r in range(cnt):
                    adds.append(("a%d[%d]" % (n, r), "sl%d[%d]" % (st, r), q, c))
                if a.kind == "vec":
                    pre.append("%s  %s *a%d_v[%d] = {%s};" %
                               (ind, t, n, cnt, ", ".join("a%d[%d]" % (n, r) for r in range(cnt))))
                    exprs.append("a%d_v" % n)
                else:
                    exprs.append("a%d[i%d]" % (n, a.idx))
        else:
            if a.kind == "ind":
                exprs.append(row_ptr(str(a.idx)))
            elif a.kind == "vec":
                pre.append("%s  %s *a%d_v[%d] = {%s};" %
                           (ind, t, n, cnt, ", ".join(row_ptr(str(r)) for r in range(cnt))))
                exprs.append("a%d_v" % n)
            else:
                exprs.append(row_ptr("i%d" % a.idx))
    return decl, pre, post, exprs, adds


def _staged_pair_passes(spec, R, used, bs, ind):
    """Passes of two elements per thread (element j * bs + threadIdx.x of
    passes j = 2m and 2m + 1): both elements' rows loaded and kernels
    evaluated before one run of colour rounds over the colours the two
    groups span (elements of one colour share no target, whichever thread
    adds them), so the two kernel bodies are independent work for the
    scheduler and the rounds and barriers are shared."""
    has_direct = any(a.kind == "direct" for a in spec.args)
    inner = ind + "  "
    L = []
    ept = R["ept"]
    for j0 in range(0, ept, 2):
        js = [j for j in (j0, j0 + 1) if j < ept]
        L.append("%sif (%d < nelem) {" % (ind, j0 * bs))
        elems = []
        for j in js:
            sfx = "_e%d" % j
            decl, pre, post, exprs, adds = _staged_element(spec, R, ind + "  ", sfx)
            elems.append((j, sfx, pre, post, exprs, adds))
            L.append("%sconst bool active%s = active_%d;" % (inner, sfx, j))
            if has_direct:
                L.append("%sconst op2b_i64 e%s = e_%d;" % (inner, sfx, j))
            for st in used:
                ar = R["stage_arity"][st]
                L.append("%sconst int sl%d%s[%d] = {%s};" % (inner, st, sfx, ar, ", ".join(
                    "sl%d_%d[%d]" % (st, j, r) for r in range(ar))))
            L += decl
        for j, sfx, pre, post, exprs, adds in elems:
            L.append("%sif (active%s) {" % (inner, sfx))
            L += pre
            L += _itspace_open(spec, inner + "  ")
            L.append(_kernel_call(spec, exprs, inner + "  " + "  " * len(spec.extents)))
            L += _itspace_close(spec, inner + "  ")
            L += post
            L.append("%s}" % inner)
        hi = "chi_%d" % js[0] if len(js) == 1 else "max(chi_%d, chi_%d)" % tuple(js)
        L.append("%sfor (int c = clo_%d; c <= %s; ++c) {" % (inner, js[0], hi))
        for j, sfx, pre, post, exprs, adds in elems:
            L.append("%s  if (col_%d == c) {" % (inner, j))
            for var, lrow, q, c in adds:
                t = R["inc_pairs"][q][2]
                L.append("%s    { const int r = %s;" % (inner, lrow))
                L.append("%s      __align__(16) %s cur[%d]; op2b_srow_load(cur, acc%d, r);" % (inner, t, c, q))
                L.append("%s      for (int k = 0; k < %d; ++k) cur[k] += %s[k];" % (inner, c, var))
                L.append("%s      op2b_srow_store(acc%d, r, cur); }" % (inner, q))
            L.append("%s  }" % inner)
        L.append("%s  __syncthreads();" % inner)
        L.append("%s}" % inner)
        L.append("%s}" % ind)
    return L


def _staged_passes(spec, R, used, bs, ind):
    """The ept passes over the block's elements: compute, then add the INC
    rows into the shared accumulators colour by colour."""
    if R.get("pair", 1) == 2:
        return _staged_pair_passes(spec, R, used, bs, ind)
    decl, pre, post, exprs, adds = _staged_element(spec, R, ind + "  ")
    has_direct = any(a.kind == "direct" for a in spec.args)
    inner = ind + "  "
    L = []
    for j in range(R["ept"]):
        L.append("%sif (%d < nelem) {" % (ind, j * bs))
        L.append("%sconst bool active = active_%d;" % (inner, j))
        if has_direct:
            L.append("%sconst op2b_i64 e = e_%d;" % (inner, j))
        for st in used:
            ar = R["stage_arity"][st]
            L.append("%sconst int sl%d[%d] = {%s};" % (inner, st, ar, ", ".join(
                "sl%d_%d[%d]" % (st, j, r) for r in range(ar))))
        L += decl
        L.append("%sif (active) {" % inner)
        L += pre
        L += _itspace_open(spec, inner + "  ")
        L.append(_kernel_call(spec, exprs, inner + "  " + "  " * len(spec.extents)))
        L += _itspace_close(spec, inner + "  ")
        L += post
        L.append("%s}" % inner)
        L.append("%sfor (int c = clo_%d; c <= chi_%d; ++c) {" % (inner, j, j))
        L.append("%s  if (col_%d == c) {" % (inner, j))
        for var, lrow, q, c in adds:
            # read-modify-write of the accumulated row with vector accesses
            # (the rows are 16-byte aligned when their size allows)
            t = R["inc_pairs"][q][2]
            L.append("%s    { const int r = %s;" % (inner, lrow))
            L.append("%s      __align__(16) %s cur[%d]; op2b_srow_load(cur, acc%d, r);" % (inner, t, c, q))
            L.append("%s      for (int k = 0; k < %d; ++k) cur[k] += %s[k];" % (inner, c, var))
            L.append("%s      op2b_srow_store(acc%d, r, cur); }" % (inner, q))
        L.append("%s  }" % inner)
        L.append("%s  __syncthreads();" % inner)
        L.append("%s}" % inner)
        L.append("%s}" % ind)
    return L


def _staged_flush(R, bs, ind):
    L = []
    for q, (slot, st, ctype, cdim) in enumerate(R["inc_pairs"]):
        L.append("%sfor (int t = threadIdx.x; t < n_s%d * %d; t += %d) {" % (ind, st, cdim, bs))
        L.append("%s  const int r = t / %d, k = t - r * %d;" % (ind, cdim, cdim))
        L.append("%s  const op2b_i64 g = tl_s%d[r];" % (ind, st))
        guard = "if (g >= 0) " if R.get("padded") else ""   # padding slots
        L.append("%s  %sop2b_atomic_add(p.d%d + g * %d + k, acc%d[op2b_srow_index<%s, %d>(r, k)]);"
                 % (ind, guard, slot, cdim, q, ctype, cdim))
        L.append("%s}" % ind)
    return L


def _staged_body(spec):
    """Indirect loop over a locality partition (op2b_region_plan_build), one
    CTA per block of the reordered set.  The block's distinct target rows
    of every READ (Dat, staged Map) pair are copied to shared memory once;
    INC rows are added into shared accumulators colour by colour (the
    plan's thread colours: no two elements of a colour share a target, so
    the adds need no atomics) and added to the Dats once per distinct
    target at the end, with global atomics since neighbouring blocks share
    targets.  WRITE/RW indirect rows are global pointers (OP2 leaves their
    conflicts to the user)."""
    bs = spec.block_size
    R = spec.region
    ns = len(R["stage_arity"])
    used = staged_used(spec)
    L = ["extern \"C\" __global__ void %s %s(const op2b_params p) {" % (_bounds(spec), stub_name(spec))]
    L.append("  extern __shared__ __align__(16) unsigned char op2b_smem[];")
    L.append("  const int blk = blockIdx.x;")
    L.append("  const int start = p.rg_boff[blk];")
    L.append("  const int nelem = p.rg_boff[blk + 1] - start;")
    L.append("  const op2b_i64 set_size = p.set_size;")
    L.append("  int smem_off = 0;")
    for st in used:
        L.append("  const int n_s%d = p.rg_tcnt[blk * %d + %d];" % (st, ns, st))
        L.append("  const int *tl_s%d = p.rg_tlist + p.rg_toff[blk * %d + %d];" % (st, ns, st))
    KR = R.get("tl_regs")
    if KR:
        # the block's target ids, row r = threadIdx.x + k * bs in register
        # k: one load each, issued with the loc rows below, reused by the
        # row copies and by the flush
        for st in used:
            for k in range(KR[st]):
                L.append("  const int tg%d_%d = threadIdx.x + %d < n_s%d ? tl_s%d[threadIdx.x + %d] : 0;"
                         % (st, k, k * bs, st, st, k * bs))
    L += _staged_prefetch(spec, R, used, bs, "  ")
    for q, (slot, st, t, c) in enumerate(R["read_pairs"]):
        L.append("  %s *rd%d = (%s *)(op2b_smem + smem_off);" % (t, q, t))
        L.append("  smem_off += (n_s%d * %d * (int)sizeof(%s) + 15) & ~15;" % (st, c, t))
    if KR:
        L += _staged_copy_rows_regs(R, used, bs, "  ", KR)
    else:
        L += _staged_copy_rows(R, used, bs, "  ", "rd%d", "n_s%d", "tl_s%d")
    for q, (slot, st, t, c) in enumerate(R["inc_pairs"]):
        L.append("  %s *acc%d = (%s *)(op2b_smem + smem_off);" % (t, q, t))
        L.append("  smem_off += (n_s%d * %d * (int)sizeof(%s) + 15) & ~15;" % (st, c, t))
        L.append("  for (int t = threadIdx.x; t < n_s%d * %d; t += %d) acc%d[t] = (%s)0;"
                 % (st, c, bs, q, t))
    if R["read_pairs"]:
        L.append("  op2b_cp_async_wait();")
    L.append("  __syncthreads();")
    _gbl_prologue(spec, L)
    L += _staged_passes(spec, R, used, bs, "  ")
    if KR:
        L += _staged_flush_regs(R, bs, "  ", KR)
    else:
        L += _staged_flush(R, bs, "  ")
    _gbl_epilogue(spec, L)
    L.append("}")
    return "\n".join(L)


def _inc_sink(spec, a, n, k, src, val, ind):
    """Add the INC row ``val`` of arg n (map position k, row address src):
    an atomic add, or in the two-phase form a store to the contribution array
    of the arg's (Dat, Map) pair."""
    if spec.mode == "lma":
        # tiles of 32 elements: for one position k a warp writes 32 adjacent
        # rows, and one element's rows stay within its tile
        return "%sop2b_store(p.ld%d + op2b_lma_index(e, %d, %d) * %d, %s);" % (
            ind, a.stage, k, spec.maps[spec.stages[a.stage][1]], a.cdim, val)
    return "%sop2b_atomic_row(%s, %s);" % (ind, src, val)


def _gathered_row(spec, a, r):
    """Row ``r`` (an int or the iteration index variable) of element e of a
    READ arg read from its gathered copy (element-major: the arity rows of
    one element next to each other)."""
    return "p.d%d + ((op2b_i64)e * %d + %s) * %d" % (a.slot, spec.maps[a.mslot], r, a.cdim)


def _atomic_element(spec, ind, ranges=None):
    """Lines computing element ``e`` of an atomic-mode (or two-phase)
    indirect loop."""
    L = []
    G = set(tuple(x) for x in spec.gathered)

    def gathered(a):
        return a.access == "READ" and (a.slot, a.mslot) in G
    used_maps = sorted({a.mslot for a in spec.args if a.kind in ("ind", "vec", "its", "mat")
                        and not gathered(a)} |
                       {a.cmslot for a in spec.args if a.kind == "mat"})
    for k in used_maps:
        ar = spec.maps[k]
        L.append("%s__align__(16) int mr%d[%d];" % (ind, k, ar))
        L.append("%sop2b_load<int, %d, true>(mr%d, p.m%d + e * %d);" % (ind, ar, k, k, ar))
    pre, post, exprs, apply = [], [], [], []
    for n, a in enumerate(spec.args):
        t, c = a.ctype, a.cdim
        if a.kind == "gbl":
            exprs.append("g%d_l" % n if a.access == "READ" else "r%d" % n)
        elif a.kind == "direct":
            exprs.append(_direct_row(a, n, "e", pre, post, ind))
        elif a.kind == "ind":
            row = (_gathered_row(spec, a, a.idx) if gathered(a) else
                   "p.d%d + (op2b_i64)mr%d[%d] * %d" % (a.slot, a.mslot, a.idx, c))
            if a.access == "INC":
                pre.append("%s__align__(16) %s a%d[%d]; op2b_zero(a%d);" % (ind, t, n, c, n))
                apply.append(_inc_sink(spec, a, n, a.idx, row, "a%d" % n, ind))
                exprs.append("a%d" % n)
            elif a.access == "READ":
                pre.append("%s__align__(16) %s a%d[%d];" % (ind, t, n, c))
                pre.append("%sop2b_load<%s, %d, %s>(a%d, %s);" % (ind, t, c, _ro(a), n, row))
                exprs.append("a%d" % n)
            else:
                exprs.append(row)
        elif a.kind in ("vec", "its"):
            cnt = a.arity if a.kind == "vec" else a.ext
            var = "i%d" % a.idx if a.kind == "its" else None
            if a.access in ("READ", "INC"):
                pre.append("%s__align__(16) %s a%d[%d][%d];" % (ind, t, n, cnt, c))
                for r in range(cnt):
                    src = (_gathered_row(spec, a, r) if gathered(a) else
                           "p.d%d + (op2b_i64)mr%d[%d] * %d" % (a.slot, a.mslot, r, c))
                    if a.access == "READ":
                        pre.append("%sop2b_load<%s, %d, %s>(a%d[%d], %s);" % (ind, t, c, _ro(a), n, r, src))
                    else:
                        pre.append("%sop2b_zero(a%d[%d]);" % (ind, n, r))
                        apply.append(_inc_sink(spec, a, n, r, src, "a%d[%d]" % (n, r), ind))
                if a.kind == "vec":
                    pre.append("%s%s *a%d_v[%d] = {%s};" %
                               (ind, t, n, cnt, ", ".join("a%d[%d]" % (n, r) for r in range(cnt))))
                    exprs.append("a%d_v" % n)
                else:
                    exprs.append("a%d[%s]" % (n, var))
            else:
                if a.kind == "vec":
                    pre.append("%s%s *a%d_v[%d] = {%s};" % (
                        ind, t, n, cnt, ", ".join("p.d%d + (op2b_i64)mr%d[%d] * %d" % (a.slot, a.mslot, r, c)
                                                   for r in range(cnt))))
                    exprs.append("a%d_v" % n)
                else:
                    exprs.append("p.d%d + (op2b_i64)mr%d[%s] * %d" % (a.slot, a.mslot, var, c))
        elif a.kind == "mat":
            e0, e1 = spec.extents[0], spec.extents[1]
            if spec.mat_per_entry:
                exprs.append("(%s (*)[1])&A%d" % (t, n))
            elif a.rm * a.cm == 1:
                pre.append("%s%s A%d[%d][%d];" % (ind, t, n, e0, e1))
                exprs.append("(%s (*)[1])&A%d[i0][i1]" % (t, n))
            else:
                pre.append("%s%s A%d[%d][%d][%d][%d];" % (ind, t, n, e0, e1, a.rm, a.cm))
                exprs.append("A%d[i0][i1]" % n)
            if not spec.mat_per_entry:
                apply += _mat_addto(spec, n, a, ind, atomic=True, lma=spec.mode == "lma")
    L += pre
    L += _itspace_open(spec, ind, ranges)
    deep = ind + "  " * len(spec.extents)
    for n, a in enumerate(spec.args):
        if a.kind == "mat":
            if spec.mat_per_entry:
                L.append("%s%s A%d = (%s)0;" % (deep, a.ctype, n, a.ctype))
            elif a.rm * a.cm == 1:
                L.append("%sA%d[i0][i1] = (%s)0;" % (deep, n, a.ctype))
            else:
                L.append("%sfor (int r = 0; r < %d; ++r) for (int c = 0; c < %d; ++c) A%d[i0][i1][r][c] = (%s)0;"
                         % (deep, a.rm, a.cm, n, a.ctype))
    L.append(_kernel_call(spec, exprs, deep))
    if spec.mat_per_entry:
        L += _mat_add_entry(spec, deep)
    L += _itspace_close(spec, ind)
    L += post
    L += apply
    return L


def _mat_add_entry(spec, ind):
    """Add the entries (i0, i1) of the loop's scalar Mat args (locals A<n>)
    into their CSR positions, read from the scatter-slot tables -- one load
    per table, shared by the Mats that alias it."""
    L = []
    loaded = set()
    for n, a in enumerate(spec.args):
        if a.kind != "mat":
            continue
        j = a.slot
        tab = spec.mat_alias[j] if spec.mat_alias else j
        ri, ci = "i%d" % a.idx, "i%d" % a.cidx
        if tab not in loaded:
            loaded.add(tab)
            if spec.mat_slots_rel:
                # the local row's word of in-row positions and the row start
                L.append("%sconst unsigned long long w%d = __ldg((const unsigned long long *)p.ms%d"
                         " + (op2b_i64)%s * p.set_size + e);" % (ind, tab, tab, ri))
                L.append("%sconst int off%d = (int)((w%d >> (8 * %s)) & 0xffull);" % (ind, tab, tab, ci))
                L.append("%sconst int pos%d = off%d == 255 ? -1 : __ldg(p.mr%d + mr%d[%s]) + off%d;"
                         % (ind, tab, tab, tab, a.mslot, ri, tab))
            else:
                L.append("%sconst int pos%d = __ldg(p.ms%d + (op2b_i64)(%s * %d + %s) * p.set_size + e);"
                         % (ind, tab, tab, ri, a.carity, ci))
            L.append("%sif (pos%d < 0) op2b_flag_missing(p.err, mr%d[%s], mr%d[%s]);"
                     % (ind, tab, a.mslot, ri, a.cmslot, ci))
        if a.access == "WRITE":
            L.append("%sif (pos%d >= 0) p.mv%d[pos%d] = A%d;" % (ind, tab, j, tab, n))
        else:
            L.append("%sif (pos%d >= 0) op2b_atomic_add(&p.mv%d[pos%d], A%d);" % (ind, tab, j, tab, n))
    return L


def batch_stub_names(spec):
    """Symbols of a batched loop: the element kernel and the Global
    finalisation kernel."""
    base = stub_name(spec) + "_batch"
    return base, base + "_fin"


class BatchLayout(object):
    """Field order of op2b_batch_params (all 8-byte fields): the per-segment
    parameter blocks, the tile list, each segment's first tile (nsegs + 1
    entries), the tile and segment counts, and one partials array per
    reducing Global slot."""

    def __init__(self, spec):
        f = ["segs", "tiles", "tile_first", "ntiles", "nsegs"]
        for j, g in enumerate(spec.gbls):
            if g[2] != "READ":
                f.append("gpart%d" % j)
        self.fields = f
        self.fmt = "<" + "Q" * len(f)
        self.nbytes = struct.calcsize(self.fmt)

    def pack(self, values):
        return struct.pack(self.fmt, *[int(values.get(n, 0)) for n in self.fields])


def _batch_body(spec):
    """A batched loop: the same stub over many instances (segments) of one
    loop signature, each with its own Sets, Maps, Dats, Mats and Globals.

    The host splits every segment into tiles of ``block_size * batch``
    consecutive elements (a tile never crosses a segment) and lists them; a
    persistent grid walks the tile list, each CTA loading the tile's segment
    parameter block and running the direct / atomic element code on the
    tile's elements.  Global reductions are reduced per tile into a partials
    array, and the finalisation kernel (one warp per segment) combines each
    segment's partials in tile order: a segment's result depends only on its
    own data and the tile size, never on the other segments in the batch."""
    bs, ept = spec.block_size, spec.batch
    names = batch_stub_names(spec)
    layout = BatchLayout(spec)
    L = ["struct op2b_batch_tile { int seg; int pad; op2b_i64 first; };",
         "struct op2b_batch_params {", "  const op2b_params *segs;",
         "  const op2b_batch_tile *tiles;", "  const op2b_i64 *tile_first;",
         "  op2b_i64 ntiles, nsegs;"]
    for n in layout.fields[5:]:
        L.append("  %s *%s;" % (spec.gbls[int(n[5:])][0], n))
    L.append("};")
    elem = _direct_element if spec.mode == "direct" else _atomic_element
    L.append("extern \"C\" __global__ void %s %s(const op2b_batch_params bp) {"
             % (_bounds(spec), names[0]))
    red = [(n, a) for n, a in enumerate(spec.args) if a.kind == "gbl" and a.access != "READ"]
    for n, a in red:
        L.append("  __shared__ %s red%d[32];" % (a.ctype, n))
    L.append("  for (op2b_i64 t = blockIdx.x; t < bp.ntiles; t += gridDim.x) {")
    L.append("    const op2b_batch_tile td = bp.tiles[t];")
    L.append("    const op2b_params p = bp.segs[td.seg];")
    pro = []
    _gbl_prologue(spec, pro)
    L += ["  " + x for x in pro]
    L.append("#pragma unroll 1")
    L.append("    for (int k = 0; k < %d; ++k) {" % ept)
    L.append("      const op2b_i64 e = td.first + threadIdx.x + (op2b_i64)k * %d;" % bs)
    L.append("      if (e < p.end) {")
    L += elem(spec, "        ")
    L.append("      }")
    L.append("    }")
    for n, a in red:
        for c in range(a.cdim):
            L.append("    { const %s v = op2b_block_reduce<%d>(r%d[%d], red%d);"
                     % (a.ctype, _RED_OP[a.access], n, c, n))
            L.append("      if (threadIdx.x == 0) bp.gpart%d[t * %d + %d] = v; }" % (a.slot, a.cdim, c))
    L.append("  }")
    L.append("}")
    # finalisation: one warp per segment, partials combined in tile order
    L.append("extern \"C\" __global__ void __launch_bounds__(256) %s(const op2b_batch_params bp) {"
             % names[1])
    L.append("  const op2b_i64 s = ((op2b_i64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;")
    L.append("  const int lane = threadIdx.x & 31;")
    L.append("  if (s >= bp.nsegs) return;")
    L.append("  const op2b_params p = bp.segs[s];")
    L.append("  const op2b_i64 t0 = bp.tile_first[s], t1 = bp.tile_first[s + 1];")
    for n, a in red:
        op = _RED_OP[a.access]
        for c in range(a.cdim):
            init = "(%s)0" % a.ctype if op == 0 else "p.g%d[%d]" % (a.slot, c)
            L.append("  { %s acc = %s;" % (a.ctype, init))
            L.append("    for (op2b_i64 t = t0 + lane; t < t1; t += 32)"
                     " acc = op2b_combine<%d>(acc, bp.gpart%d[t * %d + %d]);" % (op, a.slot, a.cdim, c))
            L.append("    acc = op2b_warp_reduce<%d>(acc);" % op)
            L.append("    if (lane == 0) p.g%d[%d] = op2b_combine<%d>(p.g%d[%d], acc); }"
                     % (a.slot, c, op, a.slot, c))
    L.append("}")
    return "\n".join(L)


def _batch_plan_body(spec):
    """A batched coloured loop: every instance (segment) carries its own
    plan (block partition of ``part_size`` elements, block colours, thread
    colours, INC staging), and each launch runs the blocks of ONE colour of
    every segment -- tiles (segment, position in the segment's blkmap) --
    so no two concurrently running blocks of a segment share a target, and
    blocks of different segments never do.  Inside a block the plan's thread
    colours order the adds (no atomics); the block's staged INC rows are
    added to the Dats at its end.  No Global reductions (their loops use the
    atomic batched form)."""
    names = batch_stub_names(spec)
    L = ["struct op2b_batch_tile { int seg; int pad; op2b_i64 first; };",
         "struct op2b_batch_params {", "  const op2b_params *segs;",
         "  const op2b_batch_tile *tiles;", "  const op2b_i64 *tile_first;",
         "  op2b_i64 ntiles, nsegs;", "};"]
    L.append("extern \"C\" __global__ void %s %s(const op2b_batch_params bp) {"
             % (_bounds(spec), names[0]))
    if spec.stages:
        L.append("  extern __shared__ __align__(16) unsigned char op2b_smem[];")
    L.append("  for (op2b_i64 t = blockIdx.x; t < bp.ntiles; t += gridDim.x) {")
    L.append("    const op2b_batch_tile td = bp.tiles[t];")
    L.append("    const op2b_params p = bp.segs[td.seg];")
    L.append("    const int blk = p.blkmap[td.first];")
    L.append("    {")
    L += ["    " + x for x in _plan_block(spec, batched=True)]
    L.append("    }")
    L.append("  }")
    L.append("}")
    return "\n".join(L)


def _owner_body(spec):
    """Owner computes: one warp per target t of the owner Map (a row node of
    the Mat, or an element of the INC Dat's set).  The warp walks t's
    incidence list (flat map positions e*arity+k in ascending order), each lane
    evaluating the kernel for one incident (e, k) and keeping only t's
    contribution; the contributions are then added into the target's value(s),
    held in registers, strictly in list order -- the order in which the
    sequential backend adds them -- and the target is written once.  No
    atomics, no colouring, deterministic."""
    bs = spec.block_size
    ow = spec.owner
    A = ow["arity"]
    L = ["extern \"C\" __global__ void %s %s(const op2b_params p) {" % (_bounds(spec), stub_name(spec))]
    _gbl_prologue(spec, L)
    L.append("  const int lane = threadIdx.x & 31;")
    L.append("  const op2b_i64 nwarps = ((op2b_i64)gridDim.x * %d) >> 5;" % bs)
    L.append("  for (op2b_i64 t = ((op2b_i64)blockIdx.x * %d + threadIdx.x) >> 5; t < p.end; t += nwarps) {" % bs)
    L.append("    const int p0 = p.inc_ptr[t], p1 = p.inc_ptr[t + 1];")
    oarg = spec.args[ow["arg"]]
    T = oarg.ctype
    if ow["kind"] == "dat":
        C = oarg.cdim
        L.append("    __align__(16) %s acc[%d];" % (T, C))
        L.append("    op2b_load<%s, %d, false>(acc, p.d%d + t * %d);" % (T, C, oarg.slot, C))
    else:
        NQ = ow["nq"]
        j = oarg.slot
        L.append("    const int r0 = p.mr%d[t], r1 = p.mr%d[t + 1];" % (j, j))
        L.append("    %s acc[%d]; int cols[%d];" % (T, NQ, NQ))
        L.append("    #pragma unroll")
        L.append("    for (int q = 0; q < %d; ++q) {" % NQ)
        L.append("      const int jj = r0 + lane + 32 * q;")
        L.append("      cols[q] = jj < r1 ? p.mc%d[jj] : -1;" % j)
        L.append("      acc[q] = jj < r1 ? p.mv%d[jj] : (%s)0;" % (j, T))
        L.append("    }")
    if ow.get("kahan"):
        n_acc = C if ow["kind"] == "dat" else ow["nq"]
        L.append("    %s comp[%d];" % (T, n_acc))
        L.append("    for (int q = 0; q < %d; ++q) comp[q] = (%s)0;" % (n_acc, T))
    if ow["kind"] == "dat":
        # one lane per incident (element, map index)
        L.append("    for (int base = p0; base < p1; base += 32) {")
        L.append("      const int ii = base + lane;")
        L.append("      const bool active = ii < p1;")
        L.append("      const int pos = active ? p.inc_list[ii] : 0;")
    else:
        # one lane per kernel call: (incident (element, row index), column index)
        E1 = spec.extents[1]
        L.append("    const int ncall = (p1 - p0) * %d;" % E1)
        L.append("    for (int base = 0; base < ncall; base += 32) {")
        L.append("      const int ci = base + lane;")
        L.append("      const bool active = ci < ncall;")
        L.append("      const int ii = p0 + ci / %d;" % E1)
        L.append("      const int call_i1 = ci - (ci / %d) * %d;" % (E1, E1))
        L.append("      const int pos = active ? p.inc_list[ii] : 0;")
    L.append("      const op2b_i64 e = pos / %d;" % A)
    L.append("      const int k = pos - (int)e * %d;" % A)
    ind = "      "
    # contribution registers
    if ow["kind"] == "dat":
        L.append("%s%s contrib[%d]; op2b_zero(contrib);" % (ind, T, oarg.cdim))
    else:
        L.append("%s%s vv = (%s)0; int vc = -2;" % (ind, T, T))
    L.append("%sif (active) {" % ind)
    ind2 = ind + "  "
    used_maps = sorted({a.mslot for a in spec.args if a.kind in ("ind", "vec", "its", "mat")} |
                       {a.cmslot for a in spec.args if a.kind == "mat"})
    for kk in used_maps:
        ar = spec.maps[kk]
        L.append("%s__align__(16) int mr%d[%d];" % (ind2, kk, ar))
        L.append("%sop2b_load<int, %d, true>(mr%d, p.m%d + e * %d);" % (ind2, ar, kk, kk, ar))
    pre, exprs, select = _owner_args(
        spec, ind2, lambda src, c: "for (int q = 0; q < %d; ++q) contrib[q] += %s[q];" % (c, src))
    L += pre
    if ow["kind"] == "dat":
        nx = len(spec.extents)
        if nx == 0:
            L.append(_kernel_call(spec, exprs, ind2))
        else:
            L.append("%sconst int i0 = k;" % ind2)
            L.append(_kernel_call(spec, exprs, ind2))
        L += select
    else:
        L.append("%sconst int i%d = k;" % (ind2, oarg.idx))
        L.append("%sconst int i%d = call_i1;" % (ind2, oarg.cidx))
        L.append("%sAloc = (%s)0;" % (ind2, T))
        L.append(_kernel_call(spec, exprs, ind2))
        L.append("%svv = Aloc; vc = mr%d[i%d];" % (ind2, oarg.cmslot, oarg.cidx))
    L.append("%s}" % ind)
    # ordered accumulation over the lanes of this chunk
    if ow["kind"] == "dat":
        L.append("%sconst int nact = min(32, p1 - base);" % ind)
    else:
        L.append("%sconst int nact = min(32, ncall - base);" % ind)
    L.append("%sfor (int l = 0; l < nact; ++l) {" % ind)
    kahan = ow.get("kahan")

    def add(dst, val, q):
        if not kahan:
            return "%s += %s;" % (dst, val)
        return ("{ %s y_ = %s - comp[%s]; %s t_ = %s + y_; comp[%s] = (t_ - %s) - y_; %s = t_; }"
                % (T, val, q, T, dst, q, dst, dst))
    if ow["kind"] == "dat":
        L.append("%s  #pragma unroll" % ind)
        L.append("%s  for (int q = 0; q < %d; ++q) { const %s v = __shfl_sync(OP2B_FULL_MASK, contrib[q], l); %s }"
                 % (ind, oarg.cdim, T, add("acc[q]", "v", "q")))
    else:
        ins = oarg.access == "WRITE"
        L.append("%s  {" % ind)
        L.append("%s    const %s v = __shfl_sync(OP2B_FULL_MASK, vv, l);" % (ind, T))
        L.append("%s    const int c = __shfl_sync(OP2B_FULL_MASK, vc, l);" % ind)
        L.append("%s    bool hit = false;" % ind)
        L.append("%s    #pragma unroll" % ind)
        if ins:
            L.append("%s    for (int q = 0; q < %d; ++q) if (cols[q] == c) { acc[q] = v; hit = true; }"
                     % (ind, ow["nq"]))
        else:
            L.append("%s    for (int q = 0; q < %d; ++q) if (cols[q] == c) { %s hit = true; }"
                     % (ind, ow["nq"], add("acc[q]", "v", "q")))
        # a column the row does not store: PETSc's NEW_NONZERO_ALLOCATION_ERR
        L.append("%s    if (!__any_sync(OP2B_FULL_MASK, hit) && lane == 0) op2b_flag_missing(p.err, (int)t, c);"
                 % ind)
        L.append("%s  }" % ind)
    L.append("%s}" % ind)
    L.append("    }")
    if ow["kind"] == "dat":
        L.append("    if (lane == 0) op2b_store(p.d%d + t * %d, acc);" % (oarg.slot, oarg.cdim))
    else:
        j = oarg.slot
        L.append("    #pragma unroll")
        L.append("    for (int q = 0; q < %d; ++q) { const int jj = r0 + lane + 32 * q; if (jj < r1) p.mv%d[jj] = acc[q]; }"
                 % (ow["nq"], j))
        L.append("    if (lane == 0 && r1 - r0 > %d) atomicCAS(p.err + 3, 0, 1);" % (32 * ow["nq"]))
    L.append("  }")
    L.append("}")
    return "\n".join(L)


def _gather_body(spec):
    """Dat INC gathered per target, one thread per target ("gather" form).

    The loop's only writes are INC into one Dat through one Map (the owner
    Map, ``owner_plan``).  Thread i takes target t = inc_order[i] (targets in
    order of first use along the locality partition's element order, so the
    threads of a warp own neighbouring targets and gather overlapping rows
    through L1) and walks t's incidence (flat positions e*arity + k, in
    increasing order): for each it evaluates the kernel for element e and
    keeps the contribution for map index k.  The target's row is read once,
    the contributions added in registers in the order the sequential
    backend adds them (element order, then map index,
    pyop2/sequential.py:55-72), optionally Kahan-compensated, and the row
    is written once: no atomics, no colouring, no shared memory.  An
    element whose targets differ is evaluated once per target."""
    bs = spec.block_size
    ow = spec.owner
    A = ow["arity"]
    oarg = spec.args[ow["arg"]]
    T, C = oarg.ctype, oarg.cdim
    kahan = ow.get("kahan")
    L = ["extern \"C\" __global__ void %s %s(const op2b_params p) {" % (_bounds(spec), stub_name(spec))]
    _gbl_prologue(spec, L)
    L.append("  for (op2b_i64 i = (op2b_i64)blockIdx.x * %d + threadIdx.x; i < p.end;"
             " i += (op2b_i64)gridDim.x * %d) {" % (bs, bs))
    L.append("    const op2b_i64 t = p.inc_order[i];")
    L.append("    const int p0 = p.inc_ptr[t], p1 = p.inc_ptr[t + 1];")
    L.append("    __align__(16) %s acc[%d];" % (T, C))
    L.append("    op2b_load<%s, %d, false>(acc, p.d%d + t * %d);" % (T, C, oarg.slot, C))
    if kahan:
        L.append("    %s comp[%d];" % (T, C))
        L.append("    for (int q = 0; q < %d; ++q) comp[q] = (%s)0;" % (C, T))

    def sink(src, c):
        if not kahan:
            return "for (int q = 0; q < %d; ++q) acc[q] += %s[q];" % (c, src)
        return ("for (int q = 0; q < %d; ++q) { %s y_ = %s[q] - comp[q]; %s t_ = acc[q] + y_;"
                " comp[q] = (t_ - acc[q]) - y_; acc[q] = t_; }" % (c, T, src, T))
    L.append("    for (int ii = p0; ii < p1; ++ii) {")
    L.append("      const int pos = p.inc_list[ii];")
    L.append("      const op2b_i64 e = pos / %d;" % A)
    L.append("      const int k = pos - (int)e * %d;" % A)
    ind2 = "      "
    used_maps = sorted({a.mslot for a in spec.args if a.kind in ("ind", "vec", "its")})
    for kk in used_maps:
        ar = spec.maps[kk]
        L.append("%s__align__(16) int mr%d[%d];" % (ind2, kk, ar))
        L.append("%sop2b_load<int, %d, true>(mr%d, p.m%d + e * %d);" % (ind2, ar, kk, kk, ar))
    pre, exprs, select = _owner_args(spec, ind2, sink)
    L += pre
    if spec.extents:
        L.append("%sconst int i0 = k;" % ind2)
    L.append(_kernel_call(spec, exprs, ind2))
    L += select
    L.append("    }")
    L.append("    op2b_store(p.d%d + t * %d, acc);" % (oarg.slot, C))
    L.append("  }")
    L.append("}")
    return "\n".join(L)


def _owner_args(spec, ind2, sink):
    """(pre, exprs, select) of one kernel evaluation of an owner-computes
    stub for element e and owner map index k: READ rows loaded through the
    element's map rows (mr<slot>), INC args of the owner Dat zeroed locals
    whose row for index k is handed to ``sink(local row expression, cdim)``
    (the line that keeps the owner's share), a Mat arg one local entry."""
    pre, exprs, select = [], [], []
    for n, a in enumerate(spec.args):
        t, c = a.ctype, a.cdim
        if a.kind == "gbl":
            exprs.append("g%d_l" % n)
        elif a.kind == "direct":
            pre.append("%s__align__(16) %s a%d[%d];" % (ind2, t, n, c))
            pre.append("%sop2b_load<%s, %d, %s>(a%d, p.d%d + e * %d);" % (ind2, t, c, _ro(a), n, a.slot, c))
            exprs.append("a%d" % n)
        elif a.kind == "ind":
            pre.append("%s__align__(16) %s a%d[%d];" % (ind2, t, n, c))
            if a.access == "INC":
                pre.append("%sop2b_zero(a%d);" % (ind2, n))
                select.append("%sif (k == %d) { %s }" % (ind2, a.idx, sink("a%d" % n, c)))
            else:
                pre.append("%sop2b_load<%s, %d, %s>(a%d, p.d%d + (op2b_i64)mr%d[%d] * %d);"
                           % (ind2, t, c, _ro(a), n, a.slot, a.mslot, a.idx, c))
            exprs.append("a%d" % n)
        elif a.kind == "vec":
            cnt = a.arity
            pre.append("%s__align__(16) %s a%d[%d][%d];" % (ind2, t, n, cnt, c))
            for r in range(cnt):
                if a.access == "INC":
                    pre.append("%sop2b_zero(a%d[%d]);" % (ind2, n, r))
                    select.append("%sif (k == %d) { %s }" % (ind2, r, sink("a%d[%d]" % (n, r), c)))
                else:
                    pre.append("%sop2b_load<%s, %d, %s>(a%d[%d], p.d%d + (op2b_i64)mr%d[%d] * %d);"
                               % (ind2, t, c, _ro(a), n, r, a.slot, a.mslot, r, c))
            pre.append("%s%s *a%d_v[%d] = {%s};" % (ind2, t, n, cnt, ", ".join("a%d[%d]" % (n, r) for r in range(cnt))))
            exprs.append("a%d_v" % n)
        elif a.kind == "its":
            if a.access == "INC":
                # 1-d iteration space: the kernel runs once, at i0 = k
                pre.append("%s__align__(16) %s a%d[%d]; op2b_zero(a%d);" % (ind2, t, n, c, n))
                select.append("%s%s" % (ind2, sink("a%d" % n, c)))
                exprs.append("a%d" % n)
            else:
                cnt = a.ext
                pre.append("%s__align__(16) %s a%d[%d][%d];" % (ind2, t, n, cnt, c))
                for r in range(cnt):
                    pre.append("%sop2b_load<%s, %d, %s>(a%d[%d], p.d%d + (op2b_i64)mr%d[%d] * %d);"
                               % (ind2, t, c, _ro(a), n, r, a.slot, a.mslot, r, c))
                exprs.append("a%d[i%d]" % (n, a.idx))
        elif a.kind == "mat":
            pre.append("%s%s Aloc;" % (ind2, t))
            exprs.append("(%s (*)[1])&Aloc" % t)
    return pre, exprs, select


def owner_plan(spec, mat_row_nnz_max=None):
    """The owner description of a loop if owner-computes applies, else None.

    Applies when the loop's only writes are (a) INC into one Dat through one
    Map ('ind' / vec-map args, or an iteration-space arg of a 1-d iteration
    space), or (b) INC or WRITE into one scalar Mat through a 2-d iteration
    space with rows on index i0 -- all other args READ, no Global reduction."""
    writers = [n for n, a in enumerate(spec.args) if a.access != "READ"]
    if not writers:
        return None
    kinds = {spec.args[n].kind for n in writers}
    if kinds == {"mat"} and len(writers) == 1:
        a = spec.args[writers[0]]
        if a.rm * a.cm != 1 or len(spec.extents) != 2 or a.idx != 0 or a.cidx != 1:
            return None
        if a.access not in ("INC", "WRITE") or mat_row_nnz_max is None or mat_row_nnz_max > 64:
            return None
        if a.ext != a.arity or a.cext != a.carity:
            return None
        return {"kind": "mat", "arg": writers[0], "arity": a.arity, "mslot": a.mslot,
                "nq": 1 if mat_row_nnz_max <= 32 else 2}
    if not kinds <= {"ind", "vec", "its"}:
        return None
    ws = [spec.args[n] for n in writers]
    if any(a.access != "INC" for a in ws):
        return None
    if len({(a.slot, a.mslot) for a in ws}) != 1:
        return None
    if any(a.kind == "its" for a in ws):
        if len(spec.extents) != 1 or len(ws) != 1 or ws[0].idx != 0 or ws[0].ext != ws[0].arity:
            return None
    elif spec.extents:
        return None
    return {"kind": "dat", "arg": writers[0], "arity": ws[0].arity, "mslot": ws[0].mslot}


def lma_capable(spec):
    """True if the two-phase form can run the loop: every INC goes to a
    float64 Dat (row of 1 to 4 values) through a Map of arity <= 64 with
    each map position at most once per (Dat, Map) pair, or to a scalar
    float64 Mat over its full local tensor; no Mat WRITE and no Global
    reduction ordering issue (Globals reduce as usual)."""
    if not any(a.kind == "mat" or (a.kind in ("ind", "vec", "its") and a.access == "INC")
               for a in spec.args):
        return False
    for st in spec.stages:
        if st[2] != "double" or not 1 <= st[3] <= 4 or len(set(st[4])) != len(st[4]):
            return False
        if spec.maps[st[1]] > 64:
            return False
    for a in spec.args:
        if a.kind == "mat":
            if (a.access != "INC" or a.ctype != "double" or a.rm * a.cm != 1
                    or (spec.extents[a.idx], spec.extents[a.cidx]) != (a.arity, a.carity)
                    or a.arity * a.carity > 64):
                return False
    return True


def atomic_capable(spec):
    """True if every INC target of the loop has a native atomic add and no
    Mat is written with WRITE (insertion needs the coloured form)."""
    ok = {"double", "float", "int", "unsigned int", "unsigned long long", "long long"}
    for a in spec.args:
        if a.kind in ("ind", "vec", "its") and a.access == "INC" and a.ctype not in ok:
            return False
        if a.kind == "mat" and (a.access != "INC" or a.ctype not in ok):
            return False
    return True


def _mat_addto(spec, n, a, ind, atomic=False, lma=False):
    """Add / insert the local tensor of Mat arg n into the CSR values
    (pyop2/host.py:145-184: scalar fields add the whole block, vector fields
    add entry by entry and skip zero values when adding)."""
    e0, e1 = spec.extents[0], spec.extents[1]
    j = a.slot
    ins = a.access == "WRITE"
    L = []
    L.append("%sfor (int i0 = 0; i0 < %d; ++i0) for (int i1 = 0; i1 < %d; ++i1) {" % (ind, e0, e1))
    ri = "i%d" % a.idx
    ci = "i%d" % a.cidx
    if lma:
        # two-phase form: the local entry goes to the contribution array at
        # k = r * ca + c; op2b_lma_reduce adds it to its CSR slot
        L.append("%s  p.lm%d[op2b_lma_index(e, %s * %d + %s, %d)] = A%d[i0][i1];"
                 % (ind, j, ri, a.carity, ci, a.arity * a.carity, n))
        L.append("%s}" % ind)
        return L
    if a.rm * a.cm == 1:
        L.append("%s  const int row = mr%d[%s], colj = mr%d[%s];" % (ind, a.mslot, ri, a.cmslot, ci))
        if spec.mat_slots:
            tab = spec.mat_alias[j] if spec.mat_alias else j
            L.append("%s  const int pos = __ldg(p.ms%d + (op2b_i64)(%s * %d + %s) * p.set_size + e);"
                     % (ind, tab, ri, a.carity, ci))
        else:
            L.append("%s  const int pos = op2b_csr_find(p.mr%d, p.mc%d, row, colj);" % (ind, j, j))
        L.append("%s  if (pos < 0) op2b_flag_missing(p.err, row, colj);" % ind)
        if ins:
            L.append("%s  else p.mv%d[pos] = A%d[i0][i1];" % (ind, j, n))
        elif atomic:
            L.append("%s  else op2b_atomic_add(&p.mv%d[pos], A%d[i0][i1]);" % (ind, j, n))
        else:
            L.append("%s  else p.mv%d[pos] += A%d[i0][i1];" % (ind, j, n))
    else:
        L.append("%s  for (int r = 0; r < %d; ++r) for (int c = 0; c < %d; ++c) {" % (ind, a.rm, a.cm))
        L.append("%s    const %s v = A%d[i0][i1][r][c];" % (ind, a.ctype, n))
        if not ins:
            L.append("%s    if (v == (%s)0) continue;" % (ind, a.ctype))
        L.append("%s    const int row = %d * mr%d[%s] + r, colj = %d * mr%d[%s] + c;"
                 % (ind, a.rm, a.mslot, ri, a.cm, a.cmslot, ci))
        L.append("%s    const int pos = op2b_csr_find(p.mr%d, p.mc%d, row, colj);" % (ind, j, j))
        L.append("%s    if (pos < 0) op2b_flag_missing(p.err, row, colj);" % ind)
        if ins:
            L.append("%s    else p.mv%d[pos] = v;" % (ind, j))
        elif atomic:
            L.append("%s    else op2b_atomic_add(&p.mv%d[pos], v);" % (ind, j))
        else:
            L.append("%s    else p.mv%d[pos] += v;" % (ind, j))
        L.append("%s  }" % ind)
    L.append("%s}" % ind)
    return L


def nvrtc_options(fmad=False, extra=()):
    opts = ["--gpu-architecture=sm_100a", "-default-device", "--std=c++17", "-lineinfo",
            "--fmad=%s" % ("true" if fmad else "false"), "-DOP2B_NVRTC=1"]
    opts += list(extra)
    return opts
