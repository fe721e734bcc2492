"""The B200 (sm_100a) CUDA backend of the OP2 API.

Replaces pyop2/cuda.py.  Objects keep their data resident in device memory
owned by libop2b200.so and move it lazily, following the reference's
DeviceDataMixin state machine (pyop2/device.py:103-183): DEVICE_UNALLOCATED,
HOST (host copy newer), DEVICE (device copy newer), BOTH.

* ``Sparsity`` is built on the GPU (op2b_sparsity_build); host copies of
  rowptr/colidx/nnz are kept for the API (pyop2/base.py:1268-1312).
* ``Mat`` values are a device CSR array assembled in place by the par_loop
  stub; ``values``/``array``/``zero``/``zero_rows`` as pyop2/cuda.py:272-301.
* ``Global`` reductions are finalised on the device; the host copy is fetched
  when ``data`` is read.
* ``par_loop`` JIT-compiles one stub per loop signature (NVRTC, cached in
  memory and on disk), builds the plan on the GPU for indirect loops (cached
  per iteration set, partition size, Maps and indices, like
  pyop2/device.py:257-303) and launches colour by colour.
"""

import ctypes as C
import hashlib
import os
import struct
import weakref

import numpy as np

from . import base, codegen, overlap
from . import halo as halo_mod
from . import configuration as cfg
from . import _lib
from ._lib import call
from .base import (INC, MAX, MIN, READ, RW, WRITE, IdentityMap, IterationIndex,  # noqa: F401
                   i)
from .exceptions import DeviceError, MapValueError
from .logger import debug
from .utils import maybe_setflags, verify_reshape

DEVICE_UNALLOCATED = 'DEVICE_UNALLOCATED'
HOST = 'HOST'
DEVICE = 'DEVICE'
BOTH = 'BOTH'

_state = {'init': False, 'sm_count': 148, 'smem_optin': 232448, 'stream': 0, 'err': None,
          'l2_bytes': 0, 'trace': None}


def _setup():
    """Load the library and initialise the device (pyop2/cuda.py:824-847)."""
    if _state['init']:
        return
    _lib.load()
    call("op2b_init", int(cfg.cfg['device']))
    sm, smem, ma, mi = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
    tot, l2 = C.c_uint64(), C.c_uint64()
    call("op2b_device_info", C.byref(sm), C.byref(smem), C.byref(ma), C.byref(mi), C.byref(tot),
         C.byref(l2))
    s = C.c_uint64()
    call("op2b_default_stream", C.byref(s))
    _state.update(init=True, sm_count=sm.value, smem_optin=smem.value, stream=s.value,
                  cc=(ma.value, mi.value), total_mem=tot.value, l2_bytes=l2.value)
    _state['err'] = DeviceBuffer(16)
    _state['err'].memset(0)
    fetch = int(cfg.cfg['l2_fetch_granularity'])
    if fetch:
        call("op2b_set_l2_fetch_granularity", fetch)
    call("op2b_set_programmatic_launch", 1 if cfg.cfg['programmatic_launch'] else 0)
    reserve = int(float(cfg.cfg['pool_reserve_gb']) * (1 << 30))
    reserve = min(reserve, tot.value // 4)
    if reserve > 0:
        # grow the stream-ordered pool once, here: the device memory it maps
        # stays in the pool (release threshold: never), so the first loops
        # of a new problem do not pay for mapping fresh memory
        buf = DeviceBuffer(reserve)
        del buf
        synchronize()


def _teardown():
    if not _state['init']:
        return
    try:
        call("op2b_stream_sync", 0)
    except DeviceError:
        pass
    ParLoop._bound_cache.clear()
    _PLAN_CACHE.clear()
    _REGION_CACHE.clear()
    _GATHER_ORDER_CACHE.clear()
    _REPLICAS.clear()
    _state['init'] = False


def device_info():
    return dict(_state)


def synchronize():
    call("op2b_stream_sync", 0)


def check_errors():
    """Raise if a stub recorded a Mat insertion outside its Sparsity (PETSc's
    NEW_NONZERO_ALLOCATION_ERR, pyop2/petsc_base.py:113-115)."""
    err = _state['err']
    if err is None:
        return
    h = np.zeros(4, dtype=np.int32)
    err.to_host(h)
    if h[0]:
        err.memset(0)
        raise MapValueError("Mat entry (%d, %d) is not in the Sparsity pattern" % (h[1], h[2]))


# ----------------------------------------------------------- device memory
class DeviceBuffer(object):
    """A block of device memory, freed (stream-ordered) with the object."""

    __slots__ = ("ptr", "nbytes", "__weakref__")

    def __init__(self, nbytes):
        if _state.get('capturing'):
            raise DeviceError("device memory requested while recording a CUDA graph: run every "
                              "loop (and create its Globals) once before capture()")
        self.nbytes = int(nbytes)
        p = C.c_uint64()
        call("op2b_malloc", C.byref(p), max(self.nbytes, 16))
        self.ptr = p.value

    def __del__(self):
        try:
            if self.ptr and _state['init'] and _lib._lib is not None:
                _lib._lib.op2b_free(self.ptr)
        except Exception:
            pass
        self.ptr = 0

    def from_host(self, arr):
        arr = np.ascontiguousarray(arr)
        assert arr.nbytes <= self.nbytes
        call("op2b_memcpy_h2d", self.ptr, arr.ctypes.data, arr.nbytes, 0)

    def to_host(self, arr):
        assert arr.flags['C_CONTIGUOUS'] and arr.nbytes <= self.nbytes
        call("op2b_memcpy_d2h", arr.ctypes.data, self.ptr, arr.nbytes, 0)

    def memset(self, value=0, nbytes=None):
        call("op2b_memset", self.ptr, value, self.nbytes if nbytes is None else nbytes, 0)


def _upload(arr):
    arr = np.ascontiguousarray(arr)
    buf = DeviceBuffer(arr.nbytes)
    buf.from_host(arr)
    return buf


def pinned_empty(shape, dtype):
    """A numpy array in pinned host memory (fast, asynchronous copies)."""
    dtype = np.dtype(dtype)
    n = int(np.prod(shape)) * dtype.itemsize
    p = C.c_uint64()
    call("op2b_host_alloc", C.byref(p), max(n, 16))
    raw = (C.c_char * max(n, 16)).from_address(p.value)
    arr = np.frombuffer(raw, dtype=np.uint8, count=n).view(dtype).reshape(shape)
    weakref.finalize(raw, _lib._lib.op2b_host_free, p.value)
    arr_holder = _PinnedHolder(arr, raw)
    return arr_holder.array


class _PinnedHolder(object):
    def __init__(self, array, raw):
        self.array = array
        self.raw = raw
        array_base = array
        while array_base.base is not None and isinstance(array_base.base, np.ndarray):
            array_base = array_base.base


# ------------------------------------------------------------------ classes
Arg = base.Arg
Set = base.Set
Halo = base.Halo
IterationSpace = base.IterationSpace


class Kernel(base.Kernel):
    """User kernel; the code is compiled for the device inside the stub."""


class DeviceDataMixin(object):
    """Host/device coherence (pyop2/device.py:103-183)."""

    DEVICE_UNALLOCATED = DEVICE_UNALLOCATED
    HOST = HOST
    DEVICE = DEVICE
    BOTH = BOTH

    @property
    def state(self):
        return self._state

    @state.setter
    def state(self, value):
        self._state = value

    @property
    def _bytes_per_elem(self):
        return self.dtype.itemsize * self.cdim

    @property
    def _is_scalar(self):
        return self.cdim == 1


class Dat(DeviceDataMixin, base.Dat):

    def __init__(self, dataset, data=None, dtype=None, name=None, soa=None, uid=None):
        base.Dat.__init__(self, dataset, data, dtype, name, soa, uid)
        self._state = DEVICE_UNALLOCATED
        self._device = None
        # write generation: bumped by every path that may change the values
        # (host write access, par_loop writes, zero, device arithmetic); READ
        # replicas compare it to know they are current
        self._wgen = 0

    # host views ---------------------------------------------------------
    @property
    def data(self):
        if self.dataset.total_size > 0 and self._data.size == 0:
            raise RuntimeError("Illegal access: no data associated with this Dat!")
        maybe_setflags(self._data, write=True)
        self._from_device()
        if self._state is not DEVICE_UNALLOCATED:
            self._state = HOST
        self._wgen += 1
        self.needs_halo_update = True
        return self._data

    @data.setter
    def data(self, value):
        maybe_setflags(self._data, write=True)
        self._data = verify_reshape(value, self.dtype, self._data.shape)
        if self._state is not DEVICE_UNALLOCATED:
            self._state = HOST
        self._wgen += 1

    @property
    def data_ro(self):
        if self.dataset.total_size > 0 and self._data.size == 0:
            raise RuntimeError("Illegal access: no data associated with this Dat!")
        maybe_setflags(self._data, write=True)
        self._from_device()
        if self._state is not DEVICE_UNALLOCATED:
            self._state = BOTH
        maybe_setflags(self._data, write=False)
        return self._data

    # device side --------------------------------------------------------
    def _allocate_device(self):
        if self._state is DEVICE_UNALLOCATED:
            self._device = DeviceBuffer(max(self._data.nbytes, 16))
            self._state = HOST

    def _to_device(self):
        self._allocate_device()
        if self._state is HOST:
            if self.soa and self.cdim > 1:
                staging = _upload(self._data)
                call("op2b_transpose", self._device.ptr, staging.ptr, self.dataset.total_size,
                     self.cdim, self.dtype.itemsize, 1, 0)
                del staging
            else:
                self._device.from_host(self._data)
            self._state = BOTH

    def _from_device(self):
        if self._state is DEVICE:
            maybe_setflags(self._data, write=True)
            if self.soa and self.cdim > 1:
                staging = DeviceBuffer(self._data.nbytes)
                call("op2b_transpose", staging.ptr, self._device.ptr, self.dataset.total_size,
                     self.cdim, self.dtype.itemsize, 0, 0)
                staging.to_host(self._data)
            else:
                self._device.to_host(self._data)
            self._state = BOTH

    @property
    def array(self):
        """Device buffer of the values (uploaded if needed)."""
        self._to_device()
        return self._device

    def zero(self):
        """Zero the Dat on the device."""
        self._allocate_device()
        self._device.memset(0)
        self._state = DEVICE
        self._wgen += 1

    # ------------------------------------------------ arithmetic on the device
    # pyop2/base.py:749-797 computed these on the host copies; here float64 /
    # float32 (and int32 except division) Dats stay on the device
    _BINOP_DTYPES = {np.dtype(np.float64): 0, np.dtype(np.float32): 1, np.dtype(np.int32): 2}
    _BINOP_CODES = {"add": 0, "sub": 1, "mul": 2, "truediv": 3}

    def _device_binop(self, other, opname, out):
        """out = self op other on the device; False if the operands need the
        host path (other dtypes, integer division, mismatched shapes)."""
        code = self._BINOP_DTYPES.get(self.dtype)
        op = self._BINOP_CODES[opname]
        if code is None or (code == 2 and op == 3):
            return False
        n = self.dataset.total_size * self.cdim
        if np.isscalar(other):
            yptr, ys = 0, float(base.as_type(other, self.dtype))
        elif isinstance(other, Dat):
            if (other.dtype != self.dtype or other.dataset.total_size * other.cdim != n
                    or other.dataset.dim != self.dataset.dim):
                # the reference's semantics: numpy broadcasting of the two
                # value arrays, whose result must fit this Dat's shape
                # (test/unit/test_linalg.py:86-100 expect ValueError)
                return False
            other._to_device()
            yptr, ys = other._device.ptr, 0.0
        else:
            return False
        self._to_device()
        if out is not self:
            out._allocate_device()
        call("op2b_vec_binop", out._device.ptr, self._device.ptr, yptr, ys, n, op, code, 0)
        out._state = DEVICE
        out._wgen += 1
        maybe_setflags(out._data, write=False)
        return True

    def _op(self, other, op):
        name = op.__name__.strip("_")
        out = Dat(self.dataset, None, self.dtype)
        if self._device_binop(other, name, out):
            return out
        return base.Dat._op(self, other, op)

    def _iop(self, other, op):
        name = op.__name__.strip("_").lstrip("i")
        if self._device_binop(other, name, self):
            return self
        return base.Dat._iop(self, other, op)

    @property
    def norm(self):
        """L2 norm of the flattened values (on the device for float64)."""
        if self.dtype != np.float64:
            return np.linalg.norm(self.data_ro)
        self._to_device()
        r = C.c_double()
        n = self.dataset.total_size * self.cdim
        call("op2b_vec_dot", self._device.ptr, self._device.ptr, n, C.byref(r), 0)
        return float(np.sqrt(r.value))


class Const(DeviceDataMixin, base.Const):
    """Global constant: a __constant__ symbol of each stub that names it,
    uploaded when its value changed (pyop2/cuda.py:303-323)."""

    # bumped whenever any Const's value may have changed: a module whose
    # symbols were synchronised at the current stamp needs no check
    _stamp = 0

    def __init__(self, dim, data=None, name=None, dtype=None):
        base.Const.__init__(self, dim, data, name, dtype)
        self._version = 0
        self._state = HOST
        Const._stamp += 1

    @property
    def data(self):
        self._version += 1
        Const._stamp += 1
        return self._data

    @data.setter
    def data(self, value):
        self._data = verify_reshape(value, self.dtype, self.dim)
        self._version += 1
        Const._stamp += 1

    def _from_device(self):
        raise RuntimeError("Copying Const %s from device not allowed" % self)


class Global(DeviceDataMixin, base.Global):

    def __init__(self, dim, data=None, dtype=None, name=None):
        base.Global.__init__(self, dim, data, dtype, name)
        self._state = DEVICE_UNALLOCATED
        self._device = None

    @property
    def data(self):
        if len(self._data) == 0:
            raise RuntimeError("Illegal access: No data associated with this Global!")
        self._from_device()
        if self._state is not DEVICE_UNALLOCATED:
            self._state = HOST
        return self._data

    @data.setter
    def data(self, value):
        self._data = verify_reshape(value, self.dtype, self.dim)
        if self._state is not DEVICE_UNALLOCATED:
            self._state = HOST

    @property
    def data_ro(self):
        self._from_device()
        if self._state is not DEVICE_UNALLOCATED:
            self._state = BOTH
        return self._data

    def _to_device(self):
        if self._state is DEVICE_UNALLOCATED:
            self._device = DeviceBuffer(max(self._data.nbytes, 16))
            self._state = HOST
        if self._state is HOST:
            data = np.ascontiguousarray(self._data)
            if data.nbytes <= 256:
                # carried in launch parameters: does not wait for the stream
                call("op2b_memcpy_h2d_small", self._device.ptr, data.ctypes.data, data.nbytes, 0)
            else:
                self._device.from_host(data)
            self._state = BOTH

    def _from_device(self):
        if self._state is DEVICE:
            self._device.to_host(self._data)
            self._state = BOTH


_MAP_DEVICE = weakref.WeakValueDictionary()


class Map(base.Map):
    """Map with device values.  Maps whose values are the same host buffer
    share one device copy (e.g. pecell / pevcell of the airfoil demo)."""

    def __init__(self, iterset, dataset, dim, values=None, name=None):
        if values is None:
            raise MapValueError("Map values must be populated.")
        base.Map.__init__(self, iterset, dataset, dim, values, name)
        self._device = None

    def _to_device(self):
        if self._device is None:
            v = self._values
            key = (v.__array_interface__['data'][0], v.nbytes)
            buf = _MAP_DEVICE.get(key)
            if buf is None or buf.nbytes != v.nbytes:
                buf = _upload(v)
                if v.nbytes:
                    _MAP_DEVICE[key] = buf
                    self._keep_values = v
            if cfg.cfg['validate_maps'] and v.size:
                bad = C.c_int64(-1)
                rc = _lib._lib.op2b_map_validate(buf.ptr, v.size, self._dataset.total_size,
                                                 C.byref(bad), 0)
                if rc != 0:
                    raise MapValueError("Map %s: value at position %d lies outside its target "
                                        "Set of size %d" % (self._name, bad.value,
                                                            self._dataset.total_size))
            self._device = buf
        return self._device


class Sparsity(base.Sparsity):
    """CSR pattern built on the device (op2b_sparsity_build)."""

    _cache = {}

    def _build(self):
        # built on the device at first use (_ensure), not at construction
        self._handle = 0
        self._host_arrays = None

    def _ensure(self):
        if self._handle:
            return
        nmaps = len(self._rmaps)
        rptr = (C.c_uint64 * nmaps)(*[m._to_device().ptr for m in self._rmaps])
        cptr = (C.c_uint64 * nmaps)(*[m._to_device().ptr for m in self._cmaps])
        rar = (C.c_int32 * nmaps)(*[m.dim for m in self._rmaps])
        car = (C.c_int32 * nmaps)(*[m.dim for m in self._cmaps])
        its = (C.c_int32 * nmaps)(*[m.iterset.size for m in self._rmaps])
        h = C.c_uint64()
        rmult, cmult = self._dims
        call("op2b_sparsity_build", rmult, cmult, self._nrows, self._ncols, nmaps, rptr, rar, cptr,
             car, its, 0, C.byref(h))
        lsize, nz = C.c_int32(), C.c_int64()
        call("op2b_sparsity_info", h.value, C.byref(lsize), C.byref(nz))
        rp, ci, nn = C.c_uint64(), C.c_uint64(), C.c_uint64()
        call("op2b_sparsity_arrays", h.value, C.byref(rp), C.byref(ci), C.byref(nn))
        self._d_rowptr_, self._d_colidx_, self._d_nnzp = rp.value, ci.value, nn.value
        self._lsize = lsize.value
        self._d_nz_ = int(nz.value)
        self._handle = h.value

    @property
    def _d_rowptr(self):
        self._ensure()
        return self._d_rowptr_

    @property
    def _d_colidx(self):
        self._ensure()
        return self._d_colidx_

    @property
    def _d_nz(self):
        self._ensure()
        return self._d_nz_

    def _slot_table(self, rmap, cmap):
        """Scatter-slot table of scalar assembly through (rmap, cmap): the
        CSR position of every element's (r, c) entry, built on the device at
        first use and kept with the Sparsity (op2b_mat_slots_build)."""
        tables = self.__dict__.setdefault("_slot_tables", {})
        key = (id(rmap), id(cmap))
        hit = tables.get(key)
        if hit is not None:
            return hit[0]
        n = rmap.iterset.size
        buf = DeviceBuffer(max(1, n * rmap.dim * cmap.dim) * 4)
        call("op2b_mat_slots_build", self._d_rowptr, self._d_colidx, rmap._to_device().ptr,
             cmap._to_device().ptr, n, rmap.dim, cmap.dim, buf.ptr, 0)
        tables[key] = (buf, rmap, cmap)
        return buf

    def _slot_table_rel(self, rmap, cmap):
        """Compact scatter-slot table (op2b_mat_slots_rel_build): per element
        and local row one 64-bit word of in-row positions, kept with the
        Sparsity."""
        tables = self.__dict__.setdefault("_slot_tables_rel", {})
        key = (id(rmap), id(cmap))
        hit = tables.get(key)
        if hit is not None:
            return hit[0]
        n = rmap.iterset.size
        buf = DeviceBuffer(max(1, n * rmap.dim) * 8)
        call("op2b_mat_slots_rel_build", self._d_rowptr, self._d_colidx, rmap._to_device().ptr,
             cmap._to_device().ptr, n, rmap.dim, cmap.dim, buf.ptr, 0)
        tables[key] = (buf, rmap, cmap)
        return buf

    def _mat_incidence(self, rmap, cmap):
        """CSR position -> the (element, r, c) local entries that add to it,
        in element order (op2b_mat_incidence_build), kept with the
        Sparsity."""
        tables = self.__dict__.setdefault("_mat_incidences", {})
        key = (id(rmap), id(cmap))
        hit = tables.get(key)
        if hit is not None:
            return hit[0]
        h = C.c_uint64()
        call("op2b_mat_incidence_build", self._d_rowptr, self._d_colidx, rmap._to_device().ptr,
             cmap._to_device().ptr, rmap.iterset.size, rmap.dim, cmap.dim, self._d_nz, 0,
             C.byref(h))
        inc = Incidence(handle=h.value)
        tables[key] = (inc, rmap, cmap)
        return inc

    def _max_row_nnz(self):
        """Largest number of stored entries in one row."""
        if getattr(self, "_max_nnz", None) is None:
            rp = self._rowptr
            self._max_nnz = int(np.diff(rp).max()) if rp.size > 1 else 0
        return self._max_nnz

    @property
    def _o_nz(self):
        return 0

    @property
    def _o_nnz(self):
        return np.zeros(0, dtype=np.int32)

    def _host(self):
        self._ensure()
        if self._host_arrays is None:
            rowptr = np.empty(self._lsize + 1, dtype=np.int32)
            colidx = np.empty(max(self._d_nz, 0), dtype=np.int32)
            nnz = np.empty(self._lsize, dtype=np.int32)
            call("op2b_memcpy_d2h", rowptr.ctypes.data, self._d_rowptr, rowptr.nbytes, 0)
            call("op2b_memcpy_d2h", colidx.ctypes.data, self._d_colidx, colidx.nbytes, 0)
            call("op2b_memcpy_d2h", nnz.ctypes.data, self._d_nnzp, nnz.nbytes, 0)
            self._host_arrays = (rowptr, colidx, nnz)
        return self._host_arrays

    @property
    def _rowptr(self):
        return self._host()[0]

    @property
    def _colidx(self):
        return self._host()[1]

    @property
    def _d_nnz(self):
        return self._host()[2]

    @property
    def rowptr(self):
        return self._rowptr

    @property
    def colidx(self):
        return self._colidx

    def __del__(self):
        # at interpreter exit the module globals may already be gone
        try:
            h = getattr(self, "_handle", 0)
            if h and _state['init'] and _lib._lib is not None:
                _lib._lib.op2b_sparsity_free(h)
        except Exception:
            pass


class Mat(DeviceDataMixin, base.Mat):
    """Device CSR values on a Sparsity."""

    def __init__(self, sparsity, dtype=None, name=None):
        base.Mat.__init__(self, sparsity, dtype, name)
        self._state = DEVICE_UNALLOCATED
        self._vals = None
        # True while every value is known to be zero (fresh or zero()ed): the
        # two-phase reduction then need not read the values
        self._is_zero = True

    def _device_values(self):
        if self._vals is None:
            self._vals = DeviceBuffer(max(self._sparsity.nz, 1) * self.dtype.itemsize)
            self._vals.memset(0)
            self._state = DEVICE
        return self._vals

    @property
    def array(self):
        """CSR values (host copy)."""
        check_errors()
        out = np.zeros(self._sparsity.nz, dtype=self.dtype)
        if self._vals is not None:
            self._vals.to_host(out)
        return out

    @property
    def values(self):
        """Dense matrix (only sensible for small matrices)."""
        rows = self._sparsity.nrows * self.dims[0]
        cols = self._sparsity.ncols * self.dims[1]
        ret = np.zeros((rows, cols), dtype=self.dtype)
        vals = self.array
        rowptr, colidx = self._sparsity._rowptr, self._sparsity._colidx
        for r in range(rows):
            ret[r, colidx[rowptr[r]:rowptr[r + 1]]] = vals[rowptr[r]:rowptr[r + 1]]
        return ret

    def zero(self):
        self._device_values().memset(0)
        self._is_zero = True

    def zero_rows(self, rows, diag_val):
        """Zero the given rows except the diagonal, set to diag_val.

        Rows are CSR row numbers.  A row outside [0, number of rows) raises
        IndexError before anything runs on the device, as PETSc's
        zeroRowsLocal does for the reference (pyop2/petsc_base.py:131-135);
        the library checks the same bound again before its launch."""
        rows = np.ascontiguousarray(np.asarray(rows, dtype=np.int64).ravel())
        self._sparsity._ensure()
        nrows = self._sparsity._lsize
        if rows.size and (rows.min() < 0 or rows.max() >= nrows):
            bad = rows[(rows < 0) | (rows >= nrows)][0]
            raise IndexError("zero_rows: row %d outside [0, %d)" % (bad, nrows))
        rows = rows.astype(np.int32)
        vals = self._device_values()
        self._is_zero = False
        call("op2b_mat_zero_rows", vals.ptr, self._sparsity._d_rowptr, self._sparsity._d_colidx,
             nrows, rows.ctypes.data_as(C.POINTER(C.c_int32)), rows.size, float(diag_val),
             self.dtype.itemsize, 0)

    def _assemble(self):
        pass


_CG_REASONS = {1: "converged (relative or absolute tolerance)", 2: "diverged (dtol)",
               3: "breakdown (non-finite residual)", 4: "iteration limit"}


class Solver(base.Solver):
    """Conjugate gradients with Jacobi or no preconditioning on the device
    (op2b_cg_solve), for the reference's defaults 'cg' + 'jacobi'
    (pyop2/base.py:1591-1601, pyop2/petsc_base.py:160-220).  Like PETSc's
    default, the solve starts from x = 0 and tests the preconditioned
    residual norm against max(rtol * r0, atol) and dtol * r0.  After a solve,
    ``iterations``, ``reason`` and ``residual_history`` describe it."""

    def solve(self, A, x, b):
        p = self.parameters
        if p['linear_solver'] != 'cg':
            raise NotImplementedError("linear_solver %r: the B200 backend solves with 'cg'"
                                      % p['linear_solver'])
        pc = p['preconditioner']
        if pc not in ('jacobi', 'none', None):
            raise NotImplementedError("preconditioner %r: the B200 backend offers 'jacobi' and "
                                      "'none'" % pc)
        check_errors()
        sp = A.sparsity
        sp._ensure()
        nrows = sp._lsize
        for d, nm in ((x, "x"), (b, "b")):
            if d.dtype != np.float64 or d.dataset.total_size * d.cdim != nrows:
                raise ValueError("%s must be a float64 Dat of %d values (the Mat's rows)" % (nm, nrows))
        b._to_device()
        if x._state is DEVICE_UNALLOCATED:
            x._allocate_device()
        vals = A._device_values()
        max_it = int(p['maximum_iterations'])
        hist = np.zeros(max_it + 1, dtype=np.float64)
        its, reason = C.c_int32(), C.c_int32()
        call("op2b_cg_solve", sp._d_rowptr, sp._d_colidx, vals.ptr, nrows, sp._d_nz,
             x._device.ptr, b._device.ptr, 1 if pc == 'jacobi' else 0,
             float(p['relative_tolerance']), float(p['absolute_tolerance']),
             float(p['divergence_tolerance']), max_it, C.byref(its), C.byref(reason),
             hist.ctypes.data_as(C.POINTER(C.c_double)), 0)
        x._state = DEVICE
        x._wgen += 1
        maybe_setflags(x._data, write=False)
        x.needs_halo_update = True
        self.iterations, self.reason = its.value, reason.value
        self.residual_history = hist[:its.value + 1].copy()
        if p.get('monitor_convergence'):
            for k, r in enumerate(self.residual_history):
                debug("%3d CG preconditioned residual norm %14.12e" % (k, r))
        if self.reason != 1:
            msg = ("CG failed to converge in %d iterations: %s (residual norm %e)"
                   % (self.iterations, _CG_REASONS.get(self.reason, self.reason),
                      self.residual_history[-1]))
            if p.get('error_on_nonconvergence', True):
                raise RuntimeError(msg)
            import warnings
            warnings.warn(msg)


def solve(M, x, b):
    """op2.solve (pyop2/op2.py: solve): M x = b with the default Solver
    parameters, on the device."""
    Solver().solve(M, x, b)


# ------------------------------------------------------------------- plans
_PLAN_CACHE = {}

_PLAN_ARRAYS = ("nelems", "offset", "ind_map", "loc_map", "ind_sizes", "ind_offs", "nindirect",
                "thrcol", "nthrcol", "blkmap", "ncolblk", "blkcol")


class DevicePlan(object):
    """A plan built on the GPU (op2b_plan_build), in plan.pyx's layout."""

    def __init__(self, set_size, part_size, stages, races, staging=True, thread_coloring=True):
        """stages: [(map, [idx...], bytes_per_elem)]; races: [([(map, idx)...], target_size)]."""
        ns = len(stages)
        smap = (C.c_uint64 * max(ns, 1))(*[m._to_device().ptr for m, _, _ in stages])
        sar = (C.c_int32 * max(ns, 1))(*[m.dim for m, _, _ in stages])
        snidx = (C.c_int32 * max(ns, 1))(*[len(ix) for _, ix, _ in stages])
        offs, flat = [], []
        for _, ix, _ in stages:
            offs.append(len(flat))
            flat += list(ix)
        soff = (C.c_int32 * max(ns, 1))(*offs)
        sidx = (C.c_int32 * max(len(flat), 1))(*flat)
        sbytes = (C.c_int32 * max(ns, 1))(*[b for _, _, b in stages])
        nr = len(races)
        rnent = (C.c_int32 * max(nr, 1))(*[len(e) for e, _ in races])
        rsize = (C.c_int32 * max(nr, 1))(*[s for _, s in races])
        ents = [x for e, _ in races for x in e]
        rmap = (C.c_uint64 * max(len(ents), 1))(*[m._to_device().ptr for m, _ in ents])
        rar = (C.c_int32 * max(len(ents), 1))(*[m.dim for m, _ in ents])
        ridx = (C.c_int32 * max(len(ents), 1))(*[ix for _, ix in ents])
        flags = (1 if staging else 0) | (2 if thread_coloring else 0)
        h = C.c_uint64()
        call("op2b_plan_build", set_size, part_size, ns, smap, sar, snidx, soff, sidx, sbytes, nr,
             rnent, rsize, rmap, rar, ridx, flags, 0, C.byref(h))
        self._handle = h.value
        nb, nc, nsh, ni, mx, ml, lr = (C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32(),
                                       C.c_int32(), C.c_int64(), C.c_int32())
        call("op2b_plan_info", self._handle, C.byref(nb), C.byref(nc), C.byref(nsh), C.byref(ni),
             C.byref(mx), C.byref(ml), C.byref(lr))
        self.nblocks, self.ncolors, self.nshared, self.ninds = nb.value, nc.value, nsh.value, ni.value
        self.max_nthrcol = mx.value
        self.part_size = part_size
        self.set_size = set_size
        ncb = (C.c_int32 * max(self.ncolors, 1))()
        call("op2b_plan_ncolblk_host", self._handle, ncb, self.ncolors)
        self.ncolblk_host = ncb
        self.max_blocks_per_color = max(list(ncb)[:self.ncolors] or [0])
        self.dptr = {}
        self.counts = {}
        for k, name in enumerate(_PLAN_ARRAYS):
            p, n = C.c_uint64(), C.c_int64()
            call("op2b_plan_array", self._handle, k, C.byref(p), C.byref(n))
            self.dptr[name] = p.value
            self.counts[name] = n.value

    def host_array(self, name):
        dtype = np.int16 if name == "loc_map" else np.int32
        out = np.zeros(self.counts[name], dtype=dtype)
        if out.size:
            call("op2b_memcpy_d2h", out.ctypes.data, self.dptr[name], out.nbytes, 0)
        return out

    def __getattr__(self, name):
        if name in _PLAN_ARRAYS:
            return self.host_array(name)
        raise AttributeError(name)

    def __del__(self):
        # at interpreter exit the module globals may already be gone
        try:
            h = getattr(self, "_handle", 0)
            if h and _state['init'] and _lib._lib is not None:
                _lib._lib.op2b_plan_free(h)
        except Exception:
            pass


_REGION_ARRAYS = ("order", "boff", "tlist", "toff", "tcnt", "loc", "thrcol", "nthrcol")
_REGION_CACHE = {}


class RegionPlan(object):
    """Locality partition of an iteration set (op2b_region_plan_build):
    regions grown through ``grow_map`` around hashed seeds (about one per
    ``region_size`` elements), cut into blocks of at most ``part_size``
    elements, with each block's distinct targets of every staged Map and
    thread colours over the targets of the staged Maps flagged in
    ``stage_inc``."""

    def __init__(self, set_size, part_size, region_size, grow_map, stage_maps, stage_inc=None,
                 bank_slots=False):
        ns = len(stage_maps)
        smap = (C.c_uint64 * max(ns, 1))(*[m._to_device().ptr for m in stage_maps])
        sar = (C.c_int32 * max(ns, 1))(*[m.dim for m in stage_maps])
        sinc = (C.c_int32 * max(ns, 1))(*[1 if (stage_inc is None or f) else 0
                                          for f in (stage_inc or [1] * ns)])
        h = C.c_uint64()
        call("op2b_region_plan_build", set_size, part_size, region_size, grow_map._to_device().ptr,
             grow_map.dim, grow_map.dataset.total_size, ns, smap, sar, sinc, 0, C.byref(h))
        self._handle = h.value
        if bank_slots:
            call("op2b_region_plan_bank_slots", self._handle, 0)
        self.bank_slots = bool(bank_slots)
        nb, nr, lv, tl, mt = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int64(), C.c_int32()
        mc = (C.c_int32 * max(ns, 1))()
        call("op2b_region_plan_info", self._handle, C.byref(nb), C.byref(nr), C.byref(lv), mc,
             C.byref(tl), C.byref(mt))
        self.nblocks, self.nregions, self.levels = nb.value, nr.value, lv.value
        self.max_nthrcol = mt.value
        self.max_count = list(mc)[:ns]
        self.set_size, self.part_size, self.nstage = set_size, part_size, ns
        self.region_size, self.stage_inc = region_size, stage_inc
        self._keep = [grow_map] + list(stage_maps)
        self.dptr, self.counts = {}, {}
        for k, name in enumerate(_REGION_ARRAYS):
            p, n = C.c_uint64(), C.c_int64()
            call("op2b_region_plan_array", self._handle, k, C.byref(p), C.byref(n))
            self.dptr[name], self.counts[name] = p.value, n.value

    def host_array(self, name):
        out = np.zeros(self.counts[name], dtype=np.int16 if name == "loc" else np.int32)
        if out.size:
            call("op2b_memcpy_d2h", out.ctypes.data, self.dptr[name], out.nbytes, 0)
        return out

    def __getattr__(self, name):
        if name in _REGION_ARRAYS:
            return self.host_array(name)
        raise AttributeError(name)

    def __del__(self):
        # at interpreter exit the module globals may already be gone
        try:
            h = getattr(self, "_handle", 0)
            if h and _state['init'] and _lib._lib is not None:
                _lib._lib.op2b_region_plan_free(h)
        except Exception:
            pass


_REPLICAS = {}


class ReadReplica(object):
    """A device copy of a Dat in order of first use through a Map, with the
    Map renumbered to match (op2b_first_use_order, op2b_rows_gather,
    op2b_map_renumber).  A loop that only reads the Dat through that Map in
    element order reads neighbouring rows for neighbouring elements.  The
    copy is refreshed from the Dat whenever the Dat's write generation
    changed since the last refresh; the renumbered Map is built once (Maps
    do not change once on the device)."""

    def __init__(self, dat, m):
        import weakref
        self.dat_ref, self.map_ref = weakref.ref(dat), weakref.ref(m)
        n = m.dataset.total_size
        self.rows = DeviceBuffer(max(dat._data.nbytes, 16))
        self.order = DeviceBuffer(max(n, 1) * 4)
        self.map = DeviceBuffer(max(m.values.size, 1) * 4)
        call("op2b_first_use_order", m._to_device().ptr, m.dim, m.iterset.total_size, 0, n,
             self.order.ptr, 0)
        call("op2b_map_renumber", self.map.ptr, m._to_device().ptr, m.iterset.total_size * m.dim,
             self.order.ptr, n, 0)
        self.wgen = None

    def ensure(self, dat):
        """Refresh the copy if the Dat changed since the last refresh."""
        if dat._state is HOST:
            dat._to_device()
        if self.wgen != dat._wgen:
            call("op2b_rows_gather", self.rows.ptr, dat._device.ptr, self.order.ptr,
                 dat.dataset.total_size, dat.dtype.itemsize * dat.cdim, 0)
            self.wgen = dat._wgen


class GatheredReplica(object):
    """A device copy of the rows a Map names, element by element: row k of
    element e at (e * arity + k).  A loop that only reads the Dat through
    that Map streams its rows in element order with no Map read and no
    dependent gather, at the price of arity copies of each row.  Refreshed
    from the Dat (one row gather through the Map) whenever the Dat's write
    generation changed since the last refresh."""

    def __init__(self, dat, m):
        import weakref
        self.dat_ref, self.map_ref = weakref.ref(dat), weakref.ref(m)
        self.n = m.iterset.total_size * m.dim
        self.rows = DeviceBuffer(max(self.n * dat.dtype.itemsize * dat.cdim, 16))
        self.wgen = None

    def ensure(self, dat):
        """Refresh the copy if the Dat changed since the last refresh."""
        if dat._state is HOST:
            dat._to_device()
        if self.wgen != dat._wgen:
            call("op2b_rows_gather", self.rows.ptr, dat._device.ptr, self.map_ref()._to_device().ptr,
                 self.n, dat.dtype.itemsize * dat.cdim, 0)
            self.wgen = dat._wgen


def gathered_replica(dat, m):
    key = ("gathered", id(dat), id(m))
    rep = _REPLICAS.get(key)
    if rep is None or rep.dat_ref() is not dat or rep.map_ref() is not m:
        for k in [k for k, r in _REPLICAS.items() if r.dat_ref() is None or r.map_ref() is None]:
            del _REPLICAS[k]
        rep = _REPLICAS[key] = GatheredReplica(dat, m)
    return rep


def read_replica(dat, m):
    key = (id(dat), id(m))
    rep = _REPLICAS.get(key)
    if rep is None or rep.dat_ref() is not dat or rep.map_ref() is not m:
        # replicas of Dats or Maps that no longer exist free their memory
        for k in [k for k, r in _REPLICAS.items() if r.dat_ref() is None or r.map_ref() is None]:
            del _REPLICAS[k]
        rep = _REPLICAS[key] = ReadReplica(dat, m)
    return rep


def replica_candidates(spec, specs, dats, maps):
    """(Dat slot, Map slot) pairs a loop can read through a READ replica:
    the Dat is read-only in the loop and read only through that Map (no
    direct access), and the Map serves no other Dat, Mat or INC arg; rows
    of a size that is a multiple of 4 bytes.  Only loops that walk their
    elements in set order (the atomic form) gain from it."""
    if spec.mode != "atomic":
        return []
    out = []
    for k in range(len(maps)):
        users = [s for s in specs if s.kind in ("ind", "vec", "its", "mat") and
                 (s.mslot == k or (s.kind == "mat" and s.cmslot == k))]
        if not users or any(s.kind == "mat" or s.access != "READ" for s in users):
            continue
        slots = {s.slot for s in users}
        if len(slots) != 1:
            continue
        j = slots.pop()
        d_uses = [s for s in specs if s.kind in ("ind", "vec", "its", "direct") and s.slot == j]
        if any(s.kind == "direct" or s.access != "READ" or s.mslot != k for s in d_uses):
            continue
        d = dats[j]
        if d.soa or (d.dtype.itemsize * d.cdim) % 4:
            continue
        out.append((j, k))
    return out


_GATHER_ORDER_CACHE = {}


def gather_order(iterset, maps, region, omap):
    """Targets of ``omap`` in order of first use along the element order of
    the loop's locality partition (op2b_first_use_order), cached per
    partition and Map: the target order of the gather form."""
    rp = region_plan(iterset, maps, region)
    key = (id(rp), id(omap))
    hit = _GATHER_ORDER_CACHE.get(key)
    if hit is not None and hit[0] is rp and hit[1] is omap:
        return hit[2]
    n = omap.dataset.size
    order = DeviceBuffer(max(n, 1) * 4)
    call("op2b_first_use_order", omap._to_device().ptr, omap.dim, iterset.size, rp.dptr["order"],
         n, order.ptr, 0)
    _GATHER_ORDER_CACHE[key] = (rp, omap, order)
    return order


def region_plan(iterset, maps, region, size=None):
    """The cached locality partition of a staged loop (over the set's first
    ``size`` elements, default all)."""
    n = iterset.size if size is None else int(size)
    ps = region["part_size"]
    rs = int(cfg.cfg['region_size']) or max(1, ps // 2)
    reps = [maps[k] for k in region["stage_maps"]]
    grow = reps[region["grow"]]
    inc = [st in region["inc_stages"] for st in range(len(reps))]
    banks = bool(cfg.cfg['staged_bank_slots'])
    key = (n, ps, rs, id(grow), tuple(id(m) for m in reps), tuple(inc), banks)
    plan = _REGION_CACHE.get(key)
    if plan is None:
        plan = _REGION_CACHE[key] = RegionPlan(n, ps, rs, grow, reps, inc, banks)
    return plan


def Plan(kernel, iset, *args, **kwargs):
    """Reference-compatible plan constructor (pyop2/device.py:305-322,
    plan.pyx:93-105): ``args`` are unwound Args, ``partition_size``,
    ``matrix_coloring``, ``staging`` and ``thread_coloring`` as in the
    reference.  Staging pairs follow the first appearance of each indirect
    (Dat, Map); race groups are the INC Dats and, with matrix colouring, the
    Mats' row Maps."""
    ps = kwargs.get('partition_size', 1)
    mc = kwargs.get('matrix_coloring', False)
    st = kwargs.get('staging', True)
    tc = kwargs.get('thread_coloring', True)
    iset = iset._iterset if isinstance(iset, base.IterationSpace) else iset
    stages, order = [], {}
    for a in args:
        if a._is_mat or not a._is_indirect:
            continue
        k = (id(a.data), id(a.map))
        if k not in order:
            order[k] = len(stages)
            stages.append([a.map, [], a.data.dtype.itemsize * a.data.cdim])
        stages[order[k]][1].append(a.idx)
    races, rorder = [], {}
    for a in args:
        if a._is_indirect_reduction:
            k = id(a.data)
            if k not in rorder:
                rorder[k] = len(races)
                races.append([[], a.data.dataset.size])
            races[rorder[k]][0].append((a.map, a.idx))
        elif mc and a._is_mat:
            k = id(a.data)
            rmap = a.map[0]
            if k not in rorder:
                rorder[k] = len(races)
                races.append([[], rmap.dataset.size])
            races[rorder[k]][0] += [(rmap, r) for r in range(rmap.dim)]
    return DevicePlan(iset.size, ps, [tuple(s) for s in stages], [tuple(r) for r in races],
                      staging=st, thread_coloring=tc)


# ---------------------------------------------------------------- incidence
class Incidence(object):
    """Target -> sorted (element, map index) list of a Map, on the device;
    or, given a handle from op2b_mat_incidence_build, CSR position -> sorted
    local entries of a Mat assembly."""

    def __init__(self, m=None, handle=None):
        if handle is None:
            h = C.c_uint64()
            call("op2b_incidence_build", m._to_device().ptr, m.iterset.size, m.dim,
                 m.dataset.total_size, 0, C.byref(h))
            handle = h.value
        self._handle = handle
        p, lst, md = C.c_uint64(), C.c_uint64(), C.c_int32()
        call("op2b_incidence_arrays", self._handle, C.byref(p), C.byref(lst), C.byref(md))
        self.ptr, self.list, self.max_degree = p.value, lst.value, md.value

    def __del__(self):
        try:
            if self._handle and _state['init']:
                _lib._lib.op2b_incidence_free(self._handle)
        except Exception:
            pass


def _incidence(m):
    inc = getattr(m, "_incidence_cache", None)
    if inc is None:
        inc = m._incidence_cache = Incidence(m)
    return inc


# --------------------------------------------------------------- JIT cache
_MODULES = {}


class _Module(object):
    def __init__(self, source, fmad, name, stub):
        opts = codegen.nvrtc_options(fmad=fmad)
        digest = hashlib.sha256((source + "\0" + " ".join(opts)).encode()).hexdigest()
        cubin = _disk_cache_get(digest)
        if cubin is None:
            arr = (C.c_char_p * len(opts))(*[o.encode() for o in opts])
            out = C.c_void_p()
            n = C.c_uint64()
            log = C.create_string_buffer(1 << 16)
            rc = _lib._lib.op2b_nvrtc_compile(source.encode(), (name + ".cu").encode(), arr,
                                              len(opts), C.byref(out), C.byref(n), log, len(log))
            if rc != 0:
                raise DeviceError("NVRTC compilation of the %s stub failed:\n%s\n--- source ---\n%s"
                                  % (name, _lib.last_error(), source[-6000:]))
            cubin = C.string_at(out.value, n.value)
            _lib._lib.op2b_cubin_free(out)
            _disk_cache_put(digest, cubin)
        self._cubin = cubin
        h = C.c_uint64()
        call("op2b_module_load", cubin, C.byref(h))
        self.handle = h.value
        self.fn = self.function(stub)
        self.smem_set = 48 * 1024
        self.const_versions = {}
        self.const_stamp = None

    def function(self, name):
        fn = C.c_uint64()
        call("op2b_module_function", self.handle, name.encode(), C.byref(fn))
        return fn.value

    def occupancy(self, fn, block, smem=0):
        """Resident CTAs per SM of a function of this module."""
        n = C.c_int32()
        call("op2b_function_occupancy", fn, block, smem, C.byref(n))
        return n.value

    def const_ptr(self, name):
        p, n = C.c_uint64(), C.c_uint64()
        call("op2b_module_global", self.handle, name.encode(), C.byref(p), C.byref(n))
        return p.value, n.value

    def ensure_smem(self, nbytes):
        if nbytes > self.smem_set:
            call("op2b_function_set_smem", self.fn, int(nbytes))
            self.smem_set = nbytes


def _disk_cache_get(digest):
    path = os.path.join(cfg.cfg['cache_dir'], digest + ".cubin")
    try:
        with open(path, "rb") as f:
            return f.read()
    except OSError:
        return None


def _disk_cache_put(digest, cubin):
    d = cfg.cfg['cache_dir']
    try:
        os.makedirs(d, exist_ok=True)
        tmp = os.path.join(d, "%s.%d.tmp" % (digest, os.getpid()))
        with open(tmp, "wb") as f:
            f.write(cubin)
        os.replace(tmp, os.path.join(d, digest + ".cubin"))
    except OSError:
        pass


def _get_module(spec):
    key = spec.key()
    mod = _MODULES.get(key)
    if mod is None:
        src, layout, stub = codegen.generate(spec)
        mod = _Module(src, spec.fmad, spec.kernel_name, stub)
        mod.layout = layout
        mod.source = src
        _MODULES[key] = mod
    return mod


# ------------------------------------------------------------------ par_loop
def _slots_usable(specs):
    """Scatter-slot tables serve a loop whose Mats are scalar and each
    assembled through one (row Map, column Map) pair."""
    pairs = {}
    for s in specs:
        if s.kind == "mat":
            if s.rm * s.cm != 1:
                return False
            pairs.setdefault(s.slot, set()).add((s.mslot, s.cmslot))
    return bool(pairs) and all(len(v) == 1 for v in pairs.values())


def mat_alias(specs, mats):
    """For each Mat slot, the first Mat slot on the same Sparsity assembled
    through the same (row Map, column Map) pair: their scatter-slot tables
    are one table, read once."""
    pair = {}
    for s in specs:
        if s.kind == "mat":
            pair.setdefault(s.slot, (s.mslot, s.cmslot))
    alias = []
    for j, m in enumerate(mats):
        same = [j0 for j0 in range(j)
                if mats[j0].sparsity is m.sparsity and pair.get(j0) == pair.get(j)]
        alias.append(same[0] if same else j)
    return tuple(alias)


def mat_slot_values(specs, maps, mats, rel=False):
    """Parameter values ms<j>: the scatter-slot table of each Mat slot (the
    compact in-row table with ``rel``)."""
    vals = {}
    for s in specs:
        if s.kind == "mat" and "ms%d" % s.slot not in vals:
            m = mats[s.slot]
            get = m.sparsity._slot_table_rel if rel else m.sparsity._slot_table
            vals["ms%d" % s.slot] = get(maps[s.mslot], maps[s.cmslot]).ptr
    return vals


def loop_spec(loop, block_size=None, fmad=None, owner_mode=None, mat_nnz_max=None,
              inc_mode=None, min_blocks=None, size=None):
    """Static description of a par_loop: the LoopSpec of its stub plus the
    unique Dats/Maps/Mats/Globals, the INC staging pairs and the plan race
    groups.  Touches no device memory (used to generate and test stubs)."""
    it = loop.it_space
    iterset = it.iterset
    nsz = iterset.size if size is None else int(size)
    extents = it.extents
    args = loop.args
    dats, dat_slot = [], {}
    maps, map_slot = [], {}
    mats, mat_slot = [], {}
    gbls = []
    specs = []
    # access summary per Dat: read-only if every use is READ
    dat_modes = {}
    for a in args:
        if a._is_dat:
            dat_modes.setdefault(id(a.data), set()).add(a.access._mode)

    def dslot(d):
        k = id(d)
        if k not in dat_slot:
            dat_slot[k] = len(dats)
            dats.append(d)
        return dat_slot[k]

    def mslot(m):
        k = id(m)
        if k not in map_slot:
            map_slot[k] = len(maps)
            maps.append(m)
        return map_slot[k]

    indirect = False
    for a in args:
        acc = a.access._mode
        if a._is_global:
            gbls.append(a.data)
            specs.append(codegen.ArgSpec(kind="gbl", access=acc, ctype=a.data.ctype,
                                         cdim=a.data.cdim, slot=len(gbls) - 1))
        elif a._is_mat:
            indirect = True
            m = a.data
            if id(m) not in mat_slot:
                mat_slot[id(m)] = len(mats)
                mats.append(m)
            rm, cm = m.dims
            if len(extents) != 2:
                raise MapValueError("A Mat argument needs a 2-d iteration space")
            specs.append(codegen.ArgSpec(
                kind="mat", access=acc, ctype=m.ctype, cdim=1, slot=mat_slot[id(m)],
                mslot=mslot(a.map[0]), cmslot=mslot(a.map[1]), idx=a.idx[0].index,
                cidx=a.idx[1].index, arity=a.map[0].dim, carity=a.map[1].dim,
                ext=extents[0], cext=extents[1], rm=rm, cm=cm))
        elif a._is_direct:
            d = a.data
            specs.append(codegen.ArgSpec(kind="direct", access=acc, ctype=d.ctype, cdim=d.cdim,
                                         slot=dslot(d), soa=bool(d.soa),
                                         ro=dat_modes[id(d)] == {"READ"}))
        else:
            indirect = True
            d = a.data
            if d.soa:
                raise NotImplementedError("SoA Dats are supported in direct loops only")
            if a.idx is None:
                kind, ix, ext = "vec", None, None
            elif isinstance(a.idx, IterationIndex):
                kind, ix = "its", a.idx.index
                if ix >= len(extents):
                    raise MapValueError("Iteration index %d outside the iteration space" % ix)
                ext = extents[ix]
            else:
                kind, ix, ext = "ind", int(a.idx), None
            specs.append(codegen.ArgSpec(kind=kind, access=acc, ctype=d.ctype, cdim=d.cdim,
                                         slot=dslot(d), mslot=mslot(a.map), idx=ix,
                                         arity=a.map.dim, ext=ext,
                                         ro=dat_modes[id(d)] == {"READ"}))
    # INC staging pairs and plan race groups (unwound like device.py:390-419)
    stages, stage_of = [], {}
    races, race_of = [], {}
    for n, (a, s) in enumerate(zip(args, specs)):
        if s.kind in ("ind", "vec", "its") and s.access == "INC":
            key = (s.slot, s.mslot)
            if key not in stage_of:
                stage_of[key] = len(stages)
                stages.append([s.slot, s.mslot, s.ctype, s.cdim, []])
            st = stages[stage_of[key]]
            unwound = [s.idx] if s.kind == "ind" else list(range(s.arity if s.kind == "vec" else s.ext))
            s.stage = stage_of[key]
            s.loc_rows = []
            for ix in unwound:
                s.loc_rows.append(len(st[4]))
                st[4].append(ix)
            rk = ("dat", s.slot)
            if rk not in race_of:
                race_of[rk] = len(races)
                races.append([[], a.data.dataset.size])
            races[race_of[rk]][0] += [(a.map, ix) for ix in unwound]
        elif s.kind == "mat":
            rk = ("mat", s.slot)
            rmap = a.map[0]
            if rk not in race_of:
                race_of[rk] = len(races)
                races.append([[], rmap.dataset.size])
            races[race_of[rk]][0] += [(rmap, r) for r in range(rmap.dim)]
    # loc_map rows are numbered over all staged pairs in order
    base_row = 0
    row_base = []
    for st in stages:
        row_base.append(base_row)
        base_row += len(st[4])
    for s in specs:
        if s.loc_rows is not None:
            s.loc_rows = [row_base[s.stage] + r for r in s.loc_rows]
    consts = [(c.name, c.ctype, c.cdim) for c in base.Const._definitions()]
    bs = int(block_size or cfg.cfg['block_size'])
    spec = codegen.LoopSpec(loop.kernel.name, loop.kernel.code, extents, specs,
                            [(d.ctype, bool(d.soa)) for d in dats], [m.dim for m in maps],
                            [m.ctype for m in mats],
                            [(g.ctype, g.cdim, s.access) for g, s in
                             zip(gbls, [s for s in specs if s.kind == "gbl"])],
                            consts, indirect,
                            [(st[0], st[1], st[2], st[3], tuple(st[4])) for st in stages],
                            bs, bool(cfg.cfg['fmad'] if fmad is None else fmad),
                            min_blocks=int(cfg.cfg['min_blocks_per_sm'] if min_blocks is None
                                           else min_blocks))
    owner = None
    om = cfg.cfg['owner_mode'] if owner_mode is None else owner_mode
    if indirect and om != 'never':
        nnz_max = mat_nnz_max
        if nnz_max is None and mats:
            nnz_max = mats[0].sparsity._max_row_nnz() if _state['init'] else 32
        owner = codegen.owner_plan(spec, nnz_max)
        if owner is not None and om == 'auto':
            # redundant kernel evaluations (one per map index of an element)
            # only pay where there are none: Mats and iteration-space INC
            w = spec.args[owner["arg"]]
            if owner["kind"] == "dat" and w.kind != "its":
                owner = None
    req = inc_mode or cfg.cfg['inc_mode']
    gather, gather_region = None, None
    if (owner is None and indirect and req == 'gather'
            and nsz >= int(cfg.cfg['staged_min_size'])):
        gather = codegen.owner_plan(spec, None)
        if gather is not None and gather["kind"] != "dat":
            gather = None
    if owner is not None:
        owner["kahan"] = bool(cfg.cfg['kahan'])
        spec.owner = owner
        spec.mode = "owner"
        indirect = False
    elif gather is not None:
        # thread per target over the owner Map's incidence, targets in
        # first-use order along the locality partition (the partition the
        # staged form would use; only its element order is used here)
        gather["kahan"] = bool(cfg.cfg['kahan'])
        spec.owner = gather
        spec.mode = "gather"
        R = _region_layout(specs, maps)
        ps = int(cfg.cfg['partition_size']) or 384
        R["part_size"] = max(1, min(ps, 16384 // max(R["stage_arity"])))
        gather_region = R
        indirect = False
    elif (indirect and req in ('staged', 'gather') and codegen.staged_capable(spec)
          and nsz >= int(cfg.cfg['staged_min_size'])):
        spec.mode = "staged"
        spec.region = R = _region_layout(specs, maps)
        if block_size is None:
            spec.block_size = bs = int(cfg.cfg['staged_block_size'])
        # blocks of at most part_size elements; the stub runs ept passes of bs
        ps = int(cfg.cfg['partition_size']) or 384
        R["part_size"] = ps = max(1, min(ps, 16384 // max(R["stage_arity"])))
        R["ept"] = (ps + bs - 1) // bs
        if int(cfg.cfg['staged_pair']) == 2:
            R["pair"] = 2
        if cfg.cfg['staged_bank_slots']:
            R["padded"] = True       # padding slots (target -1) to skip
        indirect = False   # one launch over the locality partition's blocks
    elif indirect and (inc_mode or cfg.cfg['inc_mode']) == 'lma' and codegen.lma_capable(spec):
        spec.mode = "lma"
        indirect = False   # launched like a direct loop, then reduced per target
    elif (indirect and req in ('atomic', 'staged', 'gather')
          and codegen.atomic_capable(spec)):
        spec.mode = "atomic"
        indirect = False   # launched like a direct loop: no plan
        spec.mat_slots = bool(cfg.cfg['mat_slots']) and _slots_usable(specs)
        if spec.mat_slots:
            spec.mat_alias = mat_alias(specs, mats)
            # entries added one by one (scalar Mats only; the kernel of one
            # (i0, i1) writes its own entry)
            spec.mat_per_entry = bool(cfg.cfg['mat_per_entry'])
            # compact in-row slot tables: per-entry adds, at most 8 columns
            # per element and rows of at most 254 entries
            if (spec.mat_per_entry and cfg.cfg['mat_slots_rel'] and _state['init']
                    and all(s.carity <= 8 for s in specs if s.kind == "mat")
                    and all(m.sparsity._max_row_nnz() <= 254 for m in mats)):
                spec.mat_slots_rel = True
            split = cfg.cfg['itspace_split']
            if split == "auto":
                # large local blocks (P2 6x6 and up): 3 x 2 warps per 32
                # elements measured fastest; small ones keep one thread
                split = "3x2" if len(extents) == 2 and extents[0] * extents[1] >= 36 else ""
            if (split and spec.mat_per_entry and len(extents) == 2
                    and all(s.kind == "mat" or s.access == "READ" for s in specs)):
                nr, nc = (int(v) for v in str(split).lower().split("x"))
                if 1 <= nr <= extents[0] and 1 <= nc <= extents[1] and nr * nc > 1:
                    spec.itspace_split = (nr, nc)
    if spec.mode == "direct":
        spec.direct_unroll = max(1, int(cfg.cfg['direct_unroll']))
    if (spec.mode == "atomic" and cfg.cfg['read_replicas'] and cfg.cfg['gathered_replicas']
            and nsz >= int(cfg.cfg['replica_min_size'])):
        # READ-only Dats read through one Map: a copy gathered per element
        # (no Map read, no dependent gather) while it fits the byte cap
        cap = float(cfg.cfg['gathered_max_gb']) * 1e9
        spec.gathered = tuple(
            (j, k) for j, k in replica_candidates(spec, specs, dats, maps)
            if iterset.total_size * maps[k].dim * dats[j].dtype.itemsize * dats[j].cdim <= cap)
    if (fmad is None and cfg.cfg['fmad_inc'] and not cfg.cfg['fmad']
            and spec.mode in ("staged", "atomic", "gather", "plan")
            and any(a.access == "INC" and a.kind != "gbl" for a in specs)):
        # loops whose INC sums are reassociated anyway (colour, atomic or
        # staged order): the element code may contract multiply-adds
        spec.fmad = True
    gspecs = [s for s in specs if s.kind == "gbl"]
    return dict(spec=spec, specs=specs, dats=dats, maps=maps, mats=mats, gbls=gbls,
                gbl_specs=gspecs, stages=stages, races=races, indirect=indirect,
                iterset=iterset, block_size=bs,
                gather_region=gather_region)


def _same_values(m1, m2):
    """Maps with the same target Set size, arity and values (e.g. one
    connectivity declared once per target DataSet) stage one target list."""
    if m1 is m2:
        return True
    if m1.dim != m2.dim or m1.dataset.size != m2.dataset.size or m1.iterset is not m2.iterset:
        return False
    v1, v2 = m1.values, m2.values
    if (v1.__array_interface__['data'][0] == v2.__array_interface__['data'][0]
            and v1.nbytes == v2.nbytes and v1.dtype == v2.dtype):
        return True        # one host buffer (as the demos declare pecell / pevcell)
    return np.array_equal(v1, v2)


def _region_layout(specs, maps):
    """Staged Maps of a staged loop: Map slots with the same values share
    one; loc rows numbered over the staged Maps in order; INC (Dat, staged
    Map) accumulators in order of first use; the growth Map is the INC
    Map with the most rows."""
    used = sorted({s.mslot for s in specs if s.kind in ("ind", "vec", "its")})
    reps, map_stage = [], {}
    for k in used:
        for st, r in enumerate(reps):
            if _same_values(maps[k], maps[r]):
                map_stage[k] = st
                break
        else:
            map_stage[k] = len(reps)
            reps.append(k)
    arity = [maps[r].dim for r in reps]
    row_base = [sum(arity[:st]) for st in range(len(reps))]
    pairs, reads = [], []
    grow = None
    for s in specs:
        if s.kind not in ("ind", "vec", "its"):
            continue
        st = map_stage[s.mslot]
        pr = (s.slot, st, s.ctype, s.cdim)
        if s.access == "INC":
            if pr not in pairs:
                pairs.append(pr)
            if grow is None or arity[st] > arity[grow]:
                grow = st
        elif s.access == "READ" and pr not in reads:
            reads.append(pr)
    inc_stages = sorted({st for (_, st, _, _) in pairs})
    return dict(map_stage=map_stage, stage_arity=arity, row_base=row_base, inc_pairs=pairs,
                read_pairs=reads, inc_stages=inc_stages, stage_maps=reps, grow=grow)


def _sync_consts(mod, consts):
    """Copy Const values into the module's __constant__ symbols when they
    changed since the module last saw them (Const._to_device,
    pyop2/cuda.py:314-320)."""
    stamp = (Const._stamp, base.Const._generation)
    if mod.const_stamp == stamp:
        return
    for c in consts:
        if mod.const_versions.get(c.name) != (id(c), c._version):
            ptr, nbytes = mod.const_ptr(c.name)
            arr = np.ascontiguousarray(c._data)
            if arr.nbytes != nbytes:
                raise RuntimeError("Const %s needs %d bytes, but only space for %d" %
                                   (c.name, arr.nbytes, nbytes))
            call("op2b_memcpy_h2d", ptr, arr.ctypes.data, arr.nbytes, 0)
            mod.const_versions[c.name] = (id(c), c._version)
    mod.const_stamp = stamp


class _StagedTooLarge(Exception):
    """The staged form of a loop needs more shared memory per CTA than the
    device has: the loop is bound in the atomic form instead."""


class _BoundLoop(object):
    """Everything about a par_loop that does not change between calls with
    the same objects: generated stub, plan, parameter block."""

    def __init__(self, loop, inc_mode=None, owner_mode=None, nelem=None):
        # nelem: bind to the set's first nelem elements only (the core of a
        # partitioned set, run in the staged form)
        info = loop_spec(loop, inc_mode=inc_mode, owner_mode=owner_mode, size=nelem)
        spec = info['spec']
        specs = info['specs']
        dats, maps, mats, gbls = info['dats'], info['maps'], info['mats'], info['gbls']
        stages, races, indirect = info['stages'], info['races'], info['indirect']
        iterset = info['iterset']
        args = loop.args
        self.spec = spec
        self.nelem = iterset.size if nelem is None else int(nelem)
        self.core_loop = None
        if spec.mode == "staged" and cfg.cfg['staged_tl_regs']:
            # target ids held in registers: as many per thread as the
            # partition's largest block needs
            rp0 = region_plan(iterset, maps, spec.region, self.nelem)
            bs0 = spec.block_size
            spec.region["tl_regs"] = [max(1, -(-int(c) // bs0)) for c in rp0.max_count]
        self.module = _get_module(spec)
        self.layout = self.module.layout
        self.indirect = indirect
        self.iterset = iterset
        self.partitioned = _partitioned(iterset)
        self.dats, self.maps, self.mats = dats, maps, mats
        self.gbl_specs = [s for s in specs if s.kind == "gbl"]
        self.dat_access = {}
        direct_write = {}
        for a, s in zip(args, specs):
            if a._is_dat:
                self.dat_access.setdefault(id(a.data), []).append(s.access)
                ok = (s.kind == "direct" and s.access == "WRITE"
                      and a.data.dataset.total_size == self.nelem)
                direct_write[id(a.data)] = direct_write.get(id(a.data), True) and ok
        # Dats the loop only writes, row by row over the whole set: a fresh
        # device copy needs no upload of the host values first
        self.write_only = {k for k, v in direct_write.items() if v}
        # accesses of the bound Dats and Mats (Globals vary per call) for
        # overlapped capture: atomic adds commute, other writes do not
        atomic = spec.mode in ("staged", "atomic")
        pairs = []
        for a, s in zip(args, specs):
            if s.kind == "gbl":
                continue
            if s.access == "READ":
                kind = "R"
            elif s.access == "INC" and atomic and s.kind != "direct":
                kind = "I"
            else:
                kind = "W"
            pairs.append((id(a.data), kind))
        self.accesses = overlap.loop_accesses(pairs)
        self.refs = [weakref.ref(o) for o in dats + maps + mats]
        self.consts = base.Const._definitions()
        self.block_size = info['block_size']
        bs = self.block_size
        # plan
        self.plan = None
        if indirect:
            ps = int(cfg.cfg['partition_size']) or self._default_part_size(stages)
            pkey = (iterset.size, ps,
                    tuple((id(maps[st[1]]), tuple(st[4])) for st in stages),
                    tuple((tuple((id(m), ix) for m, ix in ents), size) for ents, size in races))
            plan = _PLAN_CACHE.get(pkey)
            if plan is None:
                plan = DevicePlan(iterset.size, ps,
                                  [(maps[st[1]], st[4], np.dtype(dats[st[0]].dtype).itemsize * st[3])
                                   for st in stages],
                                  [(ents, size) for ents, size in races],
                                  staging=True, thread_coloring=True)
                plan._keep = [m for m in maps]
                _PLAN_CACHE[pkey] = plan
            self.plan = plan
            self.smem = plan.nshared
            if self.smem > _state['smem_optin']:
                raise DeviceError("par_loop %s needs %d bytes of shared memory per block; "
                                  "lower partition_size" % (loop.kernel.name, self.smem))
            self.module.ensure_smem(self.smem)
        # static parameter values
        vals = {}
        if indirect:
            p = self.plan.dptr
            vals.update(blkmap=p["blkmap"], offset=p["offset"], nelems=p["nelems"],
                        nthrcol=p["nthrcol"], thrcol=p["thrcol"], ind_map=p["ind_map"],
                        ind_sizes=p["ind_sizes"], ind_offs=p["ind_offs"], loc_map=p["loc_map"])
        for k, m in enumerate(maps):
            vals["m%d" % k] = m._to_device().ptr
        for j, m in enumerate(mats):
            vals["mv%d" % j] = m._device_values().ptr
            vals["mr%d" % j] = m.sparsity._d_rowptr
            vals["mc%d" % j] = m.sparsity._d_colidx
        if spec.mat_slots:
            vals.update(mat_slot_values(specs, maps, mats, rel=spec.mat_slots_rel))
        vals["err"] = _state['err'].ptr
        # READ replicas: (Dat slot, Dat, replica); the stub reads the copy
        # through the renumbered Map
        self.replicas = []
        for j, k in spec.gathered:
            rep = gathered_replica(dats[j], maps[k])
            vals["d%d" % j] = rep.rows.ptr
            self.replicas.append((j, dats[j], rep))
        if cfg.cfg['read_replicas'] and self.nelem >= int(cfg.cfg['replica_min_size']):
            for j, k in replica_candidates(spec, specs, dats, maps):
                if (j, k) in spec.gathered:
                    continue
                rep = read_replica(dats[j], maps[k])
                vals["m%d" % k] = rep.map.ptr
                self.replicas.append((j, dats[j], rep))
        self.vals = vals
        n = self.nelem
        self.range_end = n
        self.launch_smem = 0
        if indirect:
            self.grid = 0
            self.max_grid = self.plan.max_blocks_per_color
        elif spec.mode == "staged":
            rp = region_plan(iterset, maps, spec.region, self.nelem)
            self.region_plan = rp
            for name in _REGION_ARRAYS:
                vals["rg_" + name] = rp.dptr[name]
            self.launch_smem = codegen.staged_smem(spec, rp.max_count)
            if self.launch_smem > _state['smem_optin']:
                raise _StagedTooLarge()
            self.module.ensure_smem(self.launch_smem)
            self.grid = rp.nblocks
            self.max_grid = max(1, rp.nblocks)
        elif spec.mode == "lma":
            # two-phase INC: contribution arrays (phase 1, the stub) and the
            # incidences their reduction walks (phase 2, op2b_lma_reduce)
            self.lma = []
            self.kahan = bool(cfg.cfg['kahan'])
            n32 = (n + 31) // 32 * 32     # contribution arrays come in tiles of 32
            for j, m in enumerate(mats):
                s = next(a for a in specs if a.kind == "mat" and a.slot == j)
                rmap, cmap = maps[s.mslot], maps[s.cmslot]
                buf = DeviceBuffer(max(1, n32 * rmap.dim * cmap.dim) * 8)
                vals["lm%d" % j] = buf.ptr
                inc = m.sparsity._mat_incidence(rmap, cmap)
                self.lma.append((buf, inc, m, 1, m.sparsity._d_nz, rmap.dim * cmap.dim,
                                 (1 << (rmap.dim * cmap.dim)) - 1))
            for k, st in enumerate(stages):
                d, mp = dats[st[0]], maps[st[1]]
                buf = DeviceBuffer(max(1, n32 * mp.dim * st[3]) * 8)
                vals["ld%d" % k] = buf.ptr
                mask = 0
                for ix in st[4]:
                    mask |= 1 << ix
                self.lma.append((buf, _incidence(mp), d, st[3], mp.dataset.size, mp.dim, mask))
            self.grid = self._wave_grid(n, bs)
            self.max_grid = self.grid
        elif spec.mode == "gather":
            # one thread per target of the owner Map, in first-use order
            omap = maps[spec.owner["mslot"]]
            inc = _incidence(omap)
            order = gather_order(iterset, maps, info['gather_region'], omap)
            vals["inc_ptr"], vals["inc_list"], vals["inc_order"] = inc.ptr, inc.list, order.ptr
            self.gather_order = order
            self.range_end = omap.dataset.size
            self.grid = self._wave_grid(self.range_end, bs)
            self.max_grid = self.grid
        elif spec.mode == "atomic" and spec.itspace_split:
            nr, nc = spec.itspace_split
            self.grid = self._wave_grid(n * nr * nc, bs)
            self.max_grid = self.grid
        elif spec.mode == "owner":
            # one warp per target of the owner Map
            omap = maps[spec.owner["mslot"]]
            inc = _incidence(omap)
            vals["inc_ptr"], vals["inc_list"] = inc.ptr, inc.list
            self.range_end = omap.dataset.size
            warps = self.range_end
            self.grid = max(1, min((warps * 32 + bs - 1) // bs, _state['sm_count'] * 16)) if warps else 0
            self.max_grid = self.grid
        else:
            self.grid = self._wave_grid(n, bs)
            self.max_grid = self.grid

    @staticmethod
    def _default_part_size(stages):
        return 512

    def _wave_grid(self, n, bs):
        """Grid of a grid-stride stub: one wave of the CTAs that fit on the
        device at once (the stub's own occupancy), fewer when the set is
        smaller than that wave."""
        if not n:
            return 0
        occ = max(1, self.module.occupancy(self.module.fn, bs, 0))
        return max(1, min((n + bs - 1) // bs, occ * _state['sm_count']))

    def matches(self, loop):
        """The Dats, Maps and Mats the loop was bound to are all alive (the
        key holds their ids, which a new object could reuse otherwise)."""
        for r in self.refs:
            if r() is None:
                return False
        return True

    def _prepare(self, loop):
        """First run: device copies of the Dats, the full parameter block in a
        persistent buffer, and the bookkeeping later runs need."""
        vals = self.vals
        for j, d in enumerate(self.dats):
            if d._state is DEVICE_UNALLOCATED and id(d) in self.write_only:
                d._allocate_device()
                d._state = DEVICE
            d._to_device()
            vals["d%d" % j] = d._device.ptr
            if d.soa:
                vals["ds%d" % j] = d.dataset.total_size
        for j, d, rep in self.replicas:
            vals["d%d" % j] = rep.rows.ptr
        gargs = [k for k, a in enumerate(loop.args) if a._is_global]
        # (field offset of the Global's pointer, arg index, reducing?)
        self._gbl = []
        # reduction scratch belongs to the loop, not to the Global: launches of
        # one stream never overlap, and the last CTA leaves the counter at 0
        self._scratch = []
        for j, s in enumerate(self.gbl_specs):
            red = s.access != "READ"
            self._gbl.append((self.layout.offset("g%d" % j), gargs[j], red))
            if red:
                g = loop.args[gargs[j]].data
                part = DeviceBuffer(max(1, self.max_grid) * g.cdim * g.dtype.itemsize)
                cnt = DeviceBuffer(16)
                cnt.memset(0)
                self._scratch += [part, cnt]
                vals["gp%d" % j], vals["gc%d" % j] = part.ptr, cnt.ptr
        self._gptr = [None] * len(self._gbl)
        # reduction Globals whose value before the loop can travel in the
        # launch parameters: (flag field offset, struct format of one value)
        self._ginit = []
        for j, s in enumerate(self.gbl_specs):
            g = self.spec.gbls[j]
            if codegen.gbl_init_fields(g):
                dt = loop.args[gargs[j]].data.dtype
                fmt = ("<d" if dt == np.float64 else "<f4x" if dt == np.float32 else
                       "<q" if dt.kind == "i" else "<Q")
                self._ginit.append((self.layout.offset("gf%d" % j), fmt))
            else:
                self._ginit.append(None)
        self._gflag = [0] * len(self._gbl)
        self._written = [d for d in self.dats if any(m != "READ" for m in self.dat_access[id(d)])]
        self._reducing = [k for k, (_, _, red) in enumerate(self._gbl) if red]
        n = self.nelem
        self._buf = C.create_string_buffer(self.layout.pack(n, 0, self.range_end, vals),
                                           self.layout.nbytes)

    def run(self, loop, rng=None):
        """Run the loop over its whole set, or over elements [start, end)
        with ``rng`` (the direct and atomic forms, whose stubs walk the
        parameter block's element range)."""
        trace = _state['trace']
        if trace is None:
            self._run(loop, rng)
            return
        # overlapped capture: the chain's tail before and after this loop's
        # nodes, and what the loop reads and writes
        pre = _capture_tail()
        self._run(loop, rng)
        args = loop.args
        gbl = tuple((id(args[ai].data), "W" if red else "R") for _, ai, red in self._gbl)
        n = self.nelem if rng is None else rng[1] - rng[0]
        trace.append((pre, _capture_tail(), self.accesses + gbl, n))

    def _run(self, loop, rng=None):
        if getattr(self, "_buf", None) is None:
            self._prepare(loop)
        for d in self.dats:
            st = d._state
            if st is HOST:
                d._to_device()
            elif st is DEVICE_UNALLOCATED:
                raise DeviceError("Dat %s lost its device copy" % d.name)
        for j, d, rep in self.replicas:
            rep.ensure(d)
        buf = self._buf
        args = loop.args
        # one launch that reduces over the whole set can take a Global's value
        # from the host in its parameters (no upload before the loop)
        one_launch = rng is None and not self.indirect and not _state.get('capturing')
        for k, (off, ai, red) in enumerate(self._gbl):
            g = args[ai].data
            init = self._ginit[k]
            flag = 0
            if init is not None and one_launch and g._state in (HOST, DEVICE_UNALLOCATED):
                if g._device is None:
                    g._device = DeviceBuffer(max(g._data.nbytes, 16))
                goff, fmt = init
                for c, v in enumerate(g._data.reshape(-1)):
                    struct.pack_into(fmt, buf, goff + 8 + 8 * c, v)
                flag = 1
            else:
                g._to_device()
            if flag != self._gflag[k]:
                struct.pack_into("<q", buf, self._ginit[k][0], flag)
                self._gflag[k] = flag
            ptr = g._device.ptr
            if ptr != self._gptr[k]:
                struct.pack_into("<Q", buf, off, ptr)
                self._gptr[k] = ptr
        mod = self.module
        if self.consts:
            _sync_consts(mod, self.consts)
        n = self.nelem
        if rng is not None:
            if self.spec.mode not in ("direct", "atomic") or rng[0] < 0 or rng[1] > \
                    self.iterset.total_size:
                raise DeviceError("element range %s of a %s-form loop" % (rng, self.spec.mode))
            n = rng[1] - rng[0]
        if n == 0:
            return
        params = buf
        if self.indirect:
            plan = self.plan
            call("op2b_launch_colored", mod.fn, plan.ncolors, plan.ncolblk_host, self.block_size,
                 self.smem, 0, params, self.layout.nbytes, codegen.ParamLayout.COL_OFFSET)
        elif rng is not None:
            # the header's (start, end) for this launch only: the launch
            # copies the parameter block when it is issued
            struct.pack_into("<qq", buf, 16, rng[0], rng[1])
            try:
                call("op2b_launch", mod.fn, self.grid, self.block_size, self.launch_smem, 0,
                     params, self.layout.nbytes)
            finally:
                struct.pack_into("<qq", buf, 16, 0, self.range_end)
        else:
            call("op2b_launch", mod.fn, self.grid, self.block_size, self.launch_smem, 0, params,
                 self.layout.nbytes)
        if self.spec.mode == "lma":
            kahan = 1 if self.kahan else 0            # OP2B_LMA_KAHAN
            for buf, inc, target, cdim, ntargets, arity, mask in self.lma:
                if isinstance(target, Mat):
                    out = target._device_values().ptr
                    # Mat incidences hold contribution indices (OP2B_LMA_MAT_INDEX);
                    # a Mat known to be zero needs no read of its values
                    # (OP2B_LMA_FROM_ZERO)
                    flags = kahan | 4 | (2 if target._is_zero else 0)
                    target._is_zero = False
                else:
                    out, flags = target._device.ptr, kahan
                call("op2b_lma_reduce", out, cdim, inc.ptr, inc.list, ntargets, buf.ptr, n,
                     arity, mask, flags, 0)
        for d in self._written:
            d._state = DEVICE
            d._wgen += 1
            maybe_setflags(d._data, write=False)
        for k in self._reducing:
            args[self._gbl[k][1]].data._state = DEVICE
        for m in self.mats:
            m._state = DEVICE
            m._is_zero = False


_ENV = {"gen": None, "key": None}


def _env_key():
    """The part of a loop's cache key that the Consts and the configuration
    give, recomputed only when either changed."""
    gen = (cfg.generation(), base.Const._generation)
    if _ENV["gen"] != gen:
        _ENV["key"] = (tuple((c.name, c.dtype.str, c.cdim) for c in base.Const._definitions()),
                       (cfg.cfg['block_size'], cfg.cfg['partition_size'], cfg.cfg['fmad'],
                        cfg.cfg['min_blocks_per_sm'], cfg.cfg['inc_mode'], cfg.cfg['owner_mode'],
                        cfg.cfg['kahan'], cfg.cfg['mat_slots'], cfg.cfg['region_size'],
                        cfg.cfg['staged_min_size'], cfg.cfg['staged_block_size'],
                        cfg.cfg['mat_per_entry'], cfg.cfg['read_replicas'],
                        cfg.cfg['replica_min_size'], cfg.cfg['fmad_inc'],
                        cfg.cfg['itspace_split'], cfg.cfg['staged_tl_regs'],
                        cfg.cfg['direct_unroll'], cfg.cfg['mat_slots_rel'],
                        cfg.cfg['staged_pair'], cfg.cfg['gathered_replicas'],
                        cfg.cfg['gathered_max_gb'], cfg.cfg['staged_bank_slots']))
        _ENV["gen"] = gen
    return _ENV["key"]


def _loop_key(kernel, iterset, extents, args):
    """Cache key of a bound loop: the kernel's content, the iteration set
    and extents, and per argument the identity of its Dat / Mat and Maps,
    the index and the access mode (a Global only by type, so a fresh Global
    per call reuses the loop), plus the Consts and configuration."""
    k = [kernel.cache_key, id(iterset), extents]
    app = k.append
    for a in args:
        d = a._dat
        kind = _KEY_KIND.get(type(d))
        if kind is None:
            kind = _key_kind(type(d))
        if kind == "d":
            ix = a._idx
            if type(ix) is int or ix is None:
                app(("d", id(d), id(a._map), False, ix, a._access._mode))
            else:
                its = isinstance(ix, IterationIndex)
                app(("d", id(d), id(a._map), its, ix.index if its else ix, a._access._mode))
        elif kind == "g":
            app(("g", d.dtype.str, d.cdim, a._access._mode))
        else:
            m, ix = a._map, a._idx
            app(("m", id(d), id(m[0]), id(m[1]), ix[0].index, ix[1].index, a._access._mode))
    app(_env_key())
    return tuple(k)


_KEY_KIND = {}


def _key_kind(t):
    """'g' (Global), 'm' (Mat) or 'd' (anything else, a Dat) for an argument
    data type, remembered per type."""
    k = "g" if issubclass(t, base.Global) else "m" if issubclass(t, base.Mat) else "d"
    _KEY_KIND[t] = k
    return k


class _Args(object):
    """The argument list of a call that reuses a bound loop."""
    __slots__ = ("args",)

    def __init__(self, args):
        self.args = args


# ------------------------------------------------ partitioned sets (halos)
class _DeviceHaloBuffer(object):
    """A device buffer in the protocol of :mod:`pyop2_b200.halo` (copy,
    assign, host round trips, torch tensor view).  ``owner`` keeps the
    memory alive; a view of a Global's value passes the Global."""

    def __init__(self, ptr, nbytes, dtype, shape, owner=None):
        self.ptr, self.nbytes, self.dtype, self.shape = ptr, int(nbytes), np.dtype(dtype), shape
        self.owner = owner

    @classmethod
    def alloc(cls, nbytes, dtype, shape):
        buf = DeviceBuffer(max(int(nbytes), 16))
        return cls(buf.ptr, nbytes, dtype, shape, buf)

    def copy(self):
        out = _DeviceHaloBuffer.alloc(self.nbytes, self.dtype, self.shape)
        out.assign(self)
        return out

    def assign(self, other):
        if other.nbytes != self.nbytes:
            raise DeviceError("halo buffer of %d bytes assigned %d" % (self.nbytes, other.nbytes))
        if self.nbytes:
            call("op2b_memcpy_d2d", self.ptr, other.ptr, self.nbytes, 0)

    def to_host(self):
        out = np.empty(self.shape, self.dtype)
        if self.nbytes:
            call("op2b_memcpy_d2h", out.ctypes.data, self.ptr, self.nbytes, 0)
        return out

    def from_host(self, a):
        a = np.ascontiguousarray(np.asarray(a, dtype=self.dtype).reshape(self.shape))
        if self.nbytes:
            call("op2b_memcpy_h2d", self.ptr, a.ctypes.data, self.nbytes, 0)

    def tensor(self):
        """A torch CUDA tensor over the same memory (no copy)."""
        import torch
        n = self.nbytes // self.dtype.itemsize

        class _View(object):
            __cuda_array_interface__ = {"shape": (n,), "typestr": self.dtype.str,
                                        "data": (self.ptr, False), "version": 3,
                                        "strides": None, "stream": None}
        return torch.as_tensor(_View(), device="cuda")


class _DatRows(object):
    """Row store of a Dat on the device for halo exchanges: rows packed with
    op2b_halo_pack and unpacked with op2b_halo_unpack (an SoA Dat one
    component at a time, its buffers component-major)."""

    def __init__(self, dat):
        dat._to_device()
        self.dat = dat
        self.elem = np.dtype(dat.dtype).itemsize
        self.cdim = dat.cdim

    def _index(self, idx):
        # device copies of the Set's halo index lists, made once
        cache = self.dat.dataset.__dict__.setdefault("_halo_device_index", {})
        ent = cache.get(id(idx))
        if ent is None or ent[0] is not idx:
            a = np.ascontiguousarray(idx, dtype=np.int32)
            buf = DeviceBuffer(max(a.nbytes, 16))
            if a.nbytes:
                call("op2b_memcpy_h2d", buf.ptr, a.ctypes.data, a.nbytes, 0)
            ent = cache[id(idx)] = (idx, buf)
        return ent[1].ptr

    def _rows(self, n):
        return (n, self.cdim) if self.cdim > 1 else (n,)

    def new_buffer(self, n):
        return _DeviceHaloBuffer.alloc(n * self.cdim * self.elem, self.dat.dtype, self._rows(n))

    def _move(self, name, idx, buf):
        n = len(idx)
        d = self.dat
        if not n:
            return
        ix = self._index(idx)
        if d.soa:
            total = d.dataset.total_size
            for k in range(self.cdim):
                rows = d._device.ptr + k * total * self.elem
                part = buf.ptr + k * n * self.elem
                if name == "op2b_halo_pack":
                    call(name, part, rows, ix, n, self.elem, 0)
                else:
                    call(name, rows, part, ix, n, self.elem, 0)
        elif name == "op2b_halo_pack":
            call(name, buf.ptr, d._device.ptr, ix, n, self.cdim * self.elem, 0)
        else:
            call(name, d._device.ptr, buf.ptr, ix, n, self.cdim * self.elem, 0)

    def pack(self, idx):
        buf = self.new_buffer(len(idx))
        self._move("op2b_halo_pack", idx, buf)
        return buf

    def unpack(self, idx, buf):
        self._move("op2b_halo_unpack", idx, buf)
        d = self.dat
        d._state = DEVICE
        d._wgen += 1


def _global_value(g):
    """A Global's device value as a halo-protocol buffer."""
    g._to_device()
    return _DeviceHaloBuffer(g._device.ptr, g._data.nbytes, g.dtype, g._data.shape, g)


def torch_comm(group=None):
    """A halo communicator over a ``torch.distributed`` group (NCCL between
    GPUs, one process per GPU) whose transfers are ordered with the
    library's stream: torch's current stream is that stream while they are
    issued and waited for."""
    import torch
    s = C.c_uint64()
    call("op2b_default_stream", C.byref(s))
    return halo_mod.TorchComm(group, torch.cuda.ExternalStream(s.value))


def _partitioned(iterset):
    """The set has halo elements (sizes core < owned < exec < total, as the
    reference runs over distributed meshes)."""
    return not (iterset.core_size == iterset.size == iterset.exec_size == iterset.total_size)


def _set_comm(iterset):
    h = iterset.halo
    return h.comm if h is not None else MPI.comm


_RED_OPS = {"INC": "sum", "MIN": "min", "MAX": "max"}


def _loop_phases(bl, loop, args):
    """One par_loop over a partitioned set in the reference's order
    (pyop2/sequential.py:96-117): halo exchanges of the stale Dats an
    indirect loop reads, core elements, the exchanges' completion, the other
    owned elements, the Global all-reduces, the execute halo for loops that
    write through a Map.  A generator that yields where the rank waits for
    its peers (:func:`pyop2_b200.halo.run_lockstep` drives in-process ranks)."""
    it = bl.iterset
    if _state.get('capturing') and _set_comm(it).size > 1:
        raise DeviceError("a par_loop over a set shared with other ranks exchanges halos "
                          "through the host or NCCL and cannot be recorded into a CUDA graph")
    direct = all(a._map is None or a._map is IdentityMap for a in args)
    exchanges = []
    if not direct:
        # pyop2/base.py:197-206 and 1492-1499: every Dat arg read by an
        # indirect loop, once per Dat (the first arg clears the flag)
        for a in args:
            d = a._dat
            if (isinstance(d, base.Dat) and a._access in (READ, RW) and d.needs_halo_update
                    and d.dataset.halo is not None):
                d.needs_halo_update = False
                exchanges.append(halo_mod.DatExchange(_DatRows(d), d.dataset.halo,
                                                      d.dataset.halo.comm))
    comm = _set_comm(it)
    reductions, seen = [], set()
    for a in args:
        g = a._dat
        if isinstance(g, base.Global) and a._access in (INC, MIN, MAX) and id(g) not in seen:
            seen.add(id(g))
            reductions.append(halo_mod.GlobalReduction(_global_value(g), comm,
                                                       _RED_OPS[a._access._mode]))
    exec_halo = any(a._is_indirect_and_not_read or a._is_mat for a in args)

    def launch(start, end):
        if end <= start:
            return
        if start == 0 and end == it.core_size and bl.core_loop is not None:
            bl.core_loop.run(loop)
        else:
            bl.run(loop, (start, end))
    yield from halo_mod.loop_phases(it.sizes, launch, exchanges, reductions, direct, exec_halo)
    for a in args:
        if a._access is not READ and isinstance(a._dat, base.Dat):
            a._dat.needs_halo_update = True


def _bind(loop, iterset):
    """A new bound loop; loops over partitioned sets run element ranges, so
    they take the one-launch atomic form (no partition, plan or owner
    ordering over the whole set)."""
    if _partitioned(iterset):
        if any(isinstance(a._dat, base.Mat) for a in loop.args):
            raise NotImplementedError("Mat assembly over a partitioned set needs a distributed "
                                      "matrix; the B200 backend assembles Mats on one rank")
        bl = _BoundLoop(loop, inc_mode='atomic', owner_mode='never')
        if bl.spec.mode not in ("direct", "atomic"):
            raise NotImplementedError("par_loop %s over a partitioned set needs the %s form, "
                                      "which runs whole sets only" % (bl.spec.kernel_name,
                                                                      bl.spec.mode))
        core = iterset.core_size
        if bl.spec.mode == "atomic" and core > 0 and cfg.cfg['inc_mode'] in ('staged', 'gather'):
            # the core (most of a rank's elements) in the staged form over a
            # locality partition of its own; the other ranges stay atomic
            try:
                cb = _BoundLoop(loop, nelem=core)
            except _StagedTooLarge:
                cb = None
            if cb is not None and cb.spec.mode == "staged":
                bl.core_loop = cb
        return bl
    try:
        return _BoundLoop(loop)
    except _StagedTooLarge:
        return _BoundLoop(loop, inc_mode='atomic')


class ParLoop(base.ParLoop):

    _bound_cache = {}

    def _bound_key(self):
        return _loop_key(self.kernel, self.it_space.iterset, self.it_space.extents, self.args)

    def _bound(self):
        key = self._bound_key()
        bl = ParLoop._bound_cache.get(key)
        if bl is None or not bl.matches(self):
            bl = _bind(self, self.it_space.iterset)
            ParLoop._bound_cache[key] = bl
        return bl

    def compute(self):
        bl = self._bound()
        if _partitioned(bl.iterset):
            halo_mod.run(_loop_phases(bl, self, self.args))
            return
        bl.run(self)
        self.maybe_set_halo_update_needed()

    def phases(self):
        """The loop as a generator of phases (see :func:`_loop_phases`); a
        set without halo elements runs in one phase."""
        bl = self._bound()
        if _partitioned(bl.iterset):
            yield from _loop_phases(bl, self, self.args)
            return
        bl.run(self)
        self.maybe_set_halo_update_needed()


def par_loop(kernel, it_space, *args):
    """Run a parallel loop on the device (asynchronous; results are fetched
    when the host reads them).

    A call whose kernel, iteration space and argument objects (by identity)
    match an already bound loop runs it directly: those objects passed the
    reference's argument checks when the loop was bound, and the loop holds
    weak references that must all still be alive."""
    if isinstance(it_space, base.IterationSpace):
        iterset, extents = it_space._iterset, it_space._extents
    else:
        iterset, extents = it_space, ()
    try:
        key = _loop_key(kernel, iterset, extents, args)
    except (AttributeError, TypeError, IndexError):
        key = None   # not well-formed: the full path raises the reference's error
    bl = ParLoop._bound_cache.get(key) if key is not None else None
    if bl is not None and bl.matches(None):
        if bl.partitioned:
            halo_mod.run(_loop_phases(bl, _Args(args), args))
            return
        bl.run(_Args(args))
        # the Dats the call writes are the bound ones (same objects)
        for d in bl._written:
            d._needs_halo_update = True
        return
    ParLoop(kernel, it_space, *args).compute()


def par_loop_phases(kernel, it_space, *args):
    """:func:`par_loop` as a generator that yields where a rank of a
    partitioned run waits for its peers, so that several ranks held by one
    process (:class:`pyop2_b200.halo.LocalComm`) can be stepped together with
    :func:`pyop2_b200.halo.run_lockstep`."""
    return ParLoop(kernel, it_space, *args).phases()


class _MPIConfig(object):
    """The communicator of partitioned runs (pyop2/mpi.py:46-73): a
    :mod:`pyop2_b200.halo` communicator, set by ``op2.init(comm=...)``;
    one rank alone by default."""

    def __init__(self):
        self.comm = halo_mod.SelfComm()

    @property
    def parallel(self):
        return self.comm.size > 1


MPI = _MPIConfig()


# ------------------------------------------------ events, graphs, L2 flush
class Event(object):
    """CUDA event on the op2 stream (device-side timing)."""

    def __init__(self):
        h = C.c_uint64()
        call("op2b_event_create", C.byref(h))
        self.handle = h.value

    def record(self, node=False):
        """Record on the op2 stream; ``node``: inside b200.capture() the
        record becomes a node of the graph, timing every replay."""
        call("op2b_event_record_node" if node else "op2b_event_record", self.handle, 0)
        return self

    def synchronize(self):
        call("op2b_event_sync", self.handle)

    def query(self):
        """True once the work recorded before this event has completed."""
        d = C.c_int32()
        call("op2b_event_query", self.handle, C.byref(d))
        return bool(d.value)

    def elapsed_ms(self, later):
        ms = C.c_float()
        call("op2b_event_elapsed_ms", self.handle, later.handle, C.byref(ms))
        return ms.value

    def __del__(self):
        try:
            if self.handle and _state['init']:
                _lib._lib.op2b_event_destroy(self.handle)
        except Exception:
            pass


class Graph(object):
    """A CUDA graph of par_loops recorded by :func:`capture`."""

    def __init__(self):
        self.handle = 0
        self.segments = None

    def launch(self):
        call("op2b_graph_launch", self.handle, 0)

    def close(self):
        """Destroy the executable graph now rather than at collection."""
        if self.handle and _state['init']:
            h, self.handle = self.handle, 0
            call("op2b_graph_destroy", h)

    def __del__(self):
        try:
            if self.handle and _state['init']:
                _lib._lib.op2b_graph_destroy(self.handle)
        except Exception:
            pass


def _capture_tail():
    node = C.c_uint64()
    call("op2b_graph_capture_tail", 0, C.byref(node))
    return node.value


def _relaxed_exec(graph, trace, small_only=False):
    """Instantiate the captured chain ``graph`` with the edges between
    independent par_loops dropped (:mod:`pyop2_b200.overlap`); ``trace``
    holds per loop the chain's tail before and after its nodes, its
    accesses and its element count.  A loop of more than one node, and any
    node between loops, is a barrier.  ``small_only``: only loops over fewer
    elements than one 256-thread CTA per SM covers are relaxed; the others
    keep program order among themselves."""
    marks = [m for pre, post, _, _ in trace for m in (pre, post)]
    nm = len(marks)
    pos = (C.c_int64 * max(nm, 1))()
    nnodes = C.c_int64()
    call("op2b_graph_chain_positions", graph, (C.c_uint64 * max(nm, 1))(*marks), nm, pos,
         C.byref(nnodes))
    segs, cursor, small = [], 0, []
    limit = _state['sm_count'] * 256
    for k, (_, _, acc, n) in enumerate(trace):
        first, last = pos[2 * k] + 1, pos[2 * k + 1]
        if last < first:
            continue                      # the loop added no node
        if first < cursor:
            raise DeviceError("overlapped capture: loop %d's nodes are out of order" % k)
        if first > cursor:
            segs.append((cursor, first - 1, None))
            small.append(False)
        segs.append((first, last, acc if last == first else None))
        small.append(last == first and n < limit)
        cursor = last + 1
    if cursor < nnodes.value:
        segs.append((cursor, nnodes.value - 1, None))
        small.append(False)
    deps = overlap.dependencies([acc for _, _, acc in segs], small if small_only else None)
    ptr, idx = [0], []
    for d in deps:
        idx.extend(d)
        ptr.append(len(idx))
    ns = len(segs)
    h = C.c_uint64()
    call("op2b_graph_relax", graph, (C.c_int64 * max(ns, 1))(*[a for a, _, _ in segs]),
         (C.c_int64 * max(ns, 1))(*[b for _, b, _ in segs]), ns,
         (C.c_int32 * (ns + 1))(*ptr), (C.c_int32 * max(len(idx), 1))(*idx), C.byref(h))
    return h.value, [(acc is not None, d) for (_, _, acc), d in zip(segs, deps)]


class capture(object):
    """Record the par_loops issued inside the block into a CUDA graph instead
    of running them::

        with b200.capture() as g:
            op2.par_loop(...)
        g.launch()

    Every loop must have run once before (its stub, plan and device data
    exist), and the block must not read results on the host.

    ``overlap`` (default: the ``graph_overlap`` configuration key) lets
    loops that touch no common data in a conflicting way run side by side
    in the graph (:mod:`pyop2_b200.overlap`): ``True`` relaxes every loop,
    ``'small'`` only loops too small to fill the GPU (the others keep
    program order among themselves), ``False`` none; other device work
    recorded in the block stays in program order with everything around
    it."""

    def __init__(self, overlap=None):
        mode = cfg.cfg['graph_overlap'] if overlap is None else overlap
        if mode not in (True, False, "small"):
            raise ValueError("overlap %r (True, False or 'small')" % (mode,))
        self.overlap = bool(mode)
        self.small_only = mode == "small"

    def __enter__(self):
        self.graph = Graph()
        call("op2b_graph_begin", 0)
        _state['capturing'] = True
        _state['trace'] = [] if self.overlap else None
        return self.graph

    def __exit__(self, exc_type, exc, tb):
        _state['capturing'] = False
        trace, _state['trace'] = _state['trace'], None
        if trace is None:
            h = C.c_uint64()
            rc = _lib._lib.op2b_graph_end(0, C.byref(h))
            if exc_type is None:
                _lib.check(rc, "op2b_graph_end")
                self.graph.handle = h.value
            return False
        g = C.c_uint64()
        rc = _lib._lib.op2b_graph_end_capture(0, C.byref(g))
        if exc_type is not None:
            if rc == 0:
                _lib._lib.op2b_graph_free(g.value)
            return False
        _lib.check(rc, "op2b_graph_end_capture")
        try:
            # segments (par_loop or barrier) and the earlier segments each follows
            self.graph.handle, self.graph.segments = _relaxed_exec(g.value, trace,
                                                                    self.small_only)
        finally:
            call("op2b_graph_free", g.value)
        return False


_FLUSH = {}


def l2_flush():
    """Overwrite a buffer twice the size of L2, evicting cached data."""
    buf = _FLUSH.get('buf')
    if buf is None:
        buf = _FLUSH['buf'] = DeviceBuffer(max(2 * int(_state['l2_bytes']), 256 << 20))
    buf.memset(_FLUSH.setdefault('v', 0) & 0xff)
    _FLUSH['v'] += 1


def _global_zero(self):
    """Set the Global to zero on the device (no host round trip)."""
    if self._state is DEVICE_UNALLOCATED:
        self._device = DeviceBuffer(max(self._data.nbytes, 16))
    self._device.memset(0, self._data.nbytes)
    self._state = DEVICE


Global.zero = _global_zero
