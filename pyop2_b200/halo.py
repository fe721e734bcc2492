"""Halo exchange and cross-rank Global reductions for partitioned sets.

The reference's parallel execution (pyop2/sequential.py:96-117 with
pyop2/base.py:197-249 and 797-835): an indirect loop starts the halo
exchange of every Dat it reads whose halo is stale, runs its core elements,
waits for the exchange and writes the received rows into the halo, runs the
remaining owned elements, starts the all-reduce of its Global reductions,
runs the execute halo (loops that write through a Map), and finishes the
reductions -- so contributions of execute-halo elements never reach a
Global.  Direct loops exchange nothing.

B200 design: one process per GPU and its Dats in that GPU's memory.  The
rows a peer imports are packed on the device (``op2b_halo_pack``), sent and
received with NCCL point-to-point operations through ``torch.distributed``
(NVLink / NVSwitch; the library's stream is torch's current stream while
they are issued, so NCCL starts after the pack and the unpack waits for
NCCL), and written into the halo rows on the device (``op2b_halo_unpack``).
Globals are all-reduced with NCCL on a device copy of their value.

What is backend independent lives here: the communicators (:class:`TorchComm`
over ``torch.distributed`` -- NCCL for device buffers, gloo for host ones;
:class:`LocalComm` for several ranks' data in one process, whose messages
wait in a shared mailbox until the receiving rank asks for them), one Dat's
exchange (:class:`DatExchange`), one Global's reduction
(:class:`GlobalReduction`) and the loop order (:func:`loop_phases`).  A row
store -- a Dat's rows on the device or a host array -- packs rows into a
buffer and unpacks a buffer into rows; buffers copy, assign, and convert to
and from host arrays and torch tensors.
"""

import numpy as np


class HostBuffer(object):
    """A buffer in host memory (a contiguous numpy array)."""

    def __init__(self, arr):
        self.arr = np.ascontiguousarray(arr)

    def copy(self):
        return HostBuffer(self.arr.copy())

    def assign(self, other):
        self.arr[...] = np.asarray(other.arr).reshape(self.arr.shape)

    def to_host(self):
        return self.arr.copy()

    def from_host(self, a):
        self.arr[...] = np.asarray(a, dtype=self.arr.dtype).reshape(self.arr.shape)

    def tensor(self):
        import torch
        return torch.from_numpy(self.arr.reshape(-1))


class HostRows(object):
    """Row store over a host array [n][...] (the rows of a Dat held on the
    host, as the reference's numpy data)."""

    def __init__(self, arr):
        self.arr = arr

    def pack(self, index):
        return HostBuffer(self.arr[np.asarray(index)])

    def new_buffer(self, n):
        return HostBuffer(np.empty((n,) + self.arr.shape[1:], dtype=self.arr.dtype))

    def unpack(self, index, buf):
        self.arr[np.asarray(index)] = buf.arr.reshape((len(index),) + self.arr.shape[1:])


class Request(object):
    """Completion of a started operation; ``wait`` runs it to the end once."""

    def __init__(self, finish):
        self._finish = finish

    def wait(self):
        f, self._finish = self._finish, None
        if f is not None:
            f()


_OPS = ("sum", "min", "max")


# ------------------------------------------------------------ communicators
class SelfComm(object):
    """One process alone: nothing to exchange, reductions leave the value."""

    rank = 0
    size = 1

    def exchange(self, sends, recvs):
        if sends or recvs:
            raise RuntimeError("a single rank has no peers to exchange halo rows with")
        return Request(None)

    def allreduce(self, buf, op):
        if op not in _OPS:
            raise ValueError("reduction %r (sum, min or max)" % (op,))
        return Request(None)


class LocalGroup(object):
    """The shared mailbox of the :class:`LocalComm` ranks of one process."""

    def __init__(self, size):
        self.size = int(size)
        self.box = {}          # (src, dst, tag) -> [buffer copies]
        self.red = {}          # reduction sequence number -> {rank: host value}

    def comms(self):
        return [LocalComm(self, r) for r in range(self.size)]


class LocalComm(object):
    """Rank ``rank`` of an in-process group.  A send copies the buffer into
    the mailbox at once; a receive's ``wait`` takes the peer's message, so
    every rank must have started an exchange (or reduction) before any rank
    waits for it -- :func:`run_lockstep` drives ranks that way."""

    def __init__(self, group, rank):
        self.group, self.rank, self.size = group, int(rank), group.size
        self._nx = 0
        self._nred = 0

    def exchange(self, sends, recvs):
        tag = self._nx
        self._nx += 1
        for peer, buf in sends:
            self.group.box.setdefault((self.rank, peer, tag), []).append(buf.copy())

        def finish():
            for peer, buf in recvs:
                q = self.group.box.get((peer, self.rank, tag))
                if not q:
                    raise RuntimeError("rank %d: no message from rank %d (exchange %d)"
                                       % (self.rank, peer, tag))
                buf.assign(q.pop(0))
                if not q:
                    del self.group.box[(peer, self.rank, tag)]
        return Request(finish)

    def allreduce(self, buf, op):
        if op not in _OPS:
            raise ValueError("reduction %r (sum, min or max)" % (op,))
        seq = self._nred
        self._nred += 1
        slot = self.group.red.setdefault(seq, {"vals": {}, "done": set()})
        slot["vals"][self.rank] = buf.to_host()

        def finish():
            vals = slot["vals"]
            if len(vals) != self.size:
                raise RuntimeError("rank %d: reduction %d has %d of %d contributions"
                                   % (self.rank, seq, len(vals), self.size))
            stack = np.stack([vals[r] for r in range(self.size)])
            out = {"sum": stack.sum(axis=0), "min": stack.min(axis=0),
                   "max": stack.max(axis=0)}[op]
            buf.from_host(out)
            slot["done"].add(self.rank)
            if len(slot["done"]) == self.size:
                del self.group.red[seq]
        return Request(finish)


class TorchComm(object):
    """A ``torch.distributed`` process group: device buffers go over NCCL,
    host buffers over gloo.  ``stream`` (optional) is a torch stream that is
    made current while operations are issued and waited for (the library's
    own stream for device buffers)."""

    def __init__(self, group=None, stream=None):
        import torch.distributed as dist
        self.dist, self.group, self.stream = dist, group, stream
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self._nx = 0

    def _ctx(self):
        import contextlib
        if self.stream is None:
            return contextlib.nullcontext()
        import torch
        return torch.cuda.stream(self.stream)

    def exchange(self, sends, recvs):
        dist = self.dist
        tag = self._nx
        self._nx += 1
        ops = [dist.P2POp(dist.isend, b.tensor(), peer, self.group, tag) for peer, b in sends]
        ops += [dist.P2POp(dist.irecv, b.tensor(), peer, self.group, tag) for peer, b in recvs]
        with self._ctx():
            works = dist.batch_isend_irecv(ops) if ops else []
        # NCCL reads the send buffers on its own stream: they stay referenced
        # until the issuing stream has waited for the transfers, so that a
        # stream-ordered free cannot hand their memory to later work first
        held = [b for _, b in sends] + [b for _, b in recvs]

        def finish():
            with self._ctx():
                for w in works:
                    w.wait()
            del held[:]
        return Request(finish)

    def allreduce(self, buf, op):
        dist = self.dist
        rop = {"sum": dist.ReduceOp.SUM, "min": dist.ReduceOp.MIN, "max": dist.ReduceOp.MAX}[op]
        t = buf.tensor()
        with self._ctx():
            w = dist.all_reduce(t, op=rop, group=self.group, async_op=True)
        held = [buf]

        def finish():
            with self._ctx():
                w.wait()
            del held[:]
        return Request(finish)


# ------------------------------------------------------- exchange, reduction
class DatExchange(object):
    """The halo exchange of one Dat's rows (pyop2/base.py:797-835): pack the
    rows each peer imports, send them, receive the peers' rows, and unpack
    them into the halo once the receives complete."""

    def __init__(self, rows, halo, comm):
        self.rows, self.halo, self.comm = rows, halo, comm

    def begin(self):
        sends = [(q, self.rows.pack(idx)) for q, idx in enumerate(self.halo.sends) if len(idx)]
        recvs = [(q, self.rows.new_buffer(len(idx))) for q, idx in enumerate(self.halo.receives)
                 if len(idx)]
        req = self.comm.exchange(sends, recvs)

        def finish():
            req.wait()
            for q, buf in recvs:
                self.rows.unpack(self.halo.receives[q], buf)
        return Request(finish)


class GlobalReduction(object):
    """One Global's all-reduce across ranks (pyop2/base.py:216-249): the
    value reduced into a copy, which replaces the value when finished (so
    what the execute halo adds in between is dropped)."""

    def __init__(self, value, comm, op):
        self.value, self.comm, self.op = value, comm, op

    def begin(self):
        scratch = self.value.copy()
        req = self.comm.allreduce(scratch, self.op)

        def finish():
            req.wait()
            self.value.assign(scratch)
        return Request(finish)


def loop_phases(sizes, launch, exchanges=(), reductions=(), direct=False, exec_halo=False):
    """One par_loop over a partitioned set in the reference's order, as a
    generator that yields where a rank waits for its peers (run it to the
    end with :func:`run`, or several in-process ranks with
    :func:`run_lockstep`).  ``launch(start, end)`` runs elements
    [start, end); ``sizes`` = (core, owned, exec, total)."""
    core, size, exec_size = int(sizes[0]), int(sizes[1]), int(sizes[2])
    if direct:
        launch(0, size)
        red = [r.begin() for r in reductions]
        yield
        for r in red:
            r.wait()
        return
    pending = [x.begin() for x in exchanges]
    launch(0, core)
    yield
    for p in pending:
        p.wait()
    if not reductions:
        # nothing is reduced between the owned elements and the execute
        # halo: one launch covers both
        launch(core, exec_size if exec_halo else size)
        return
    launch(core, size)
    red = [r.begin() for r in reductions]
    yield
    if exec_halo:
        launch(size, exec_size)
    for r in red:
        r.wait()


def run(phases):
    """Run one rank's phases to the end (its peers run in other processes)."""
    for _ in phases:
        pass


def run_lockstep(per_rank):
    """Run the phase generators of several in-process ranks step by step:
    every rank reaches a wait point before any rank goes past it."""
    live = list(per_rank)
    while live:
        live = [g for g in live if next(g, StopIteration) is not StopIteration]
