"""Backend-independent OP2 data model.

The classes keep the API and semantics of pyop2/base.py so that user programs
written against the reference run unchanged: access descriptors (:56-90),
``Arg`` and its predicates (:94-259), ``Set`` with core/owned/exec/total sizes
(:261-400), ``IterationSpace`` (:507-564), ``Dat`` (:612-855), ``Const``
(:857-926), ``Global`` (:928-977), ``IterationIndex`` / ``i`` (:981-1016),
``Map`` / ``IdentityMap`` (:1018-1128), ``Sparsity`` (:1130-1312), ``Mat``
(:1314-1395), ``Kernel`` (:1399-1436), the ``JITModule`` cache key
(:1438-1471), ``ParLoop.check_args`` and friends (:1473-1589) and ``Solver``
parameters (:1591-1657).  Device behaviour lives in :mod:`pyop2_b200.b200`.
"""

import math
import operator
from hashlib import md5

import numpy as np

from .backends import _BackendSelector, _make_object
from .caching import Cached
from .exceptions import (DataTypeError, DimTypeError, IndexTypeError,
                         IndexValueError, MapTypeError, MapValueError, ModeValueError,
                         NameTypeError, SetTypeError, SizeTypeError, SparsityTypeError)
from .utils import as_tuple, as_type, maybe_setflags, validate_in, validate_type, verify_reshape


# --------------------------------------------------------------- access modes
class Access(object):
    """OP2 access type of an :class:`Arg`.  Use the predefined values."""

    _modes = ["READ", "WRITE", "RW", "INC", "MIN", "MAX"]

    @validate_in(('mode', _modes, ModeValueError))
    def __init__(self, mode):
        self._mode = mode

    def __str__(self):
        return "OP2 Access: %s" % self._mode

    def __repr__(self):
        return "Access('%s')" % self._mode


READ = Access("READ")
WRITE = Access("WRITE")
RW = Access("RW")
INC = Access("INC")
MIN = Access("MIN")
MAX = Access("MAX")


# ------------------------------------------------------------------------ Arg
def _new_arg(data, map, idx, access):
    """The selected backend's Arg (as ``_make_object('Arg', ...)``), built
    with positional arguments: this runs for every argument of every
    par_loop call."""
    cls = _BackendSelector._backend.__dict__.get('Arg')
    if cls is None:
        return _make_object('Arg', data=data, map=map, idx=idx, access=access)
    return cls(data, map, idx, access)


class Arg(object):
    """An argument to a :func:`par_loop`; build it by calling a Dat/Mat/Global."""

    def __init__(self, data=None, map=None, idx=None, access=None):
        self._dat = data
        self._map = map
        self._idx = idx
        self._access = access

    def __str__(self):
        return "OP2 Arg: dat %s, map %s, index %s, access %s" % \
            (self._dat, self._map, self._idx, self._access)

    def __repr__(self):
        return "Arg(%r, %r, %r, %r)" % (self._dat, self._map, self._idx, self._access)

    @property
    def ctype(self):
        return self.data.ctype

    @property
    def dtype(self):
        return self.data.dtype

    @property
    def map(self):
        return self._map

    @property
    def idx(self):
        return self._idx

    @property
    def access(self):
        return self._access

    @property
    def data(self):
        return self._dat

    @property
    def _is_soa(self):
        return self._is_dat and self._dat.soa

    @property
    def _is_vec_map(self):
        return self._is_indirect and self._idx is None

    @property
    def _is_mat(self):
        return isinstance(self._dat, Mat)

    @property
    def _is_global(self):
        return isinstance(self._dat, Global)

    @property
    def _is_global_reduction(self):
        return self._is_global and self._access in [INC, MIN, MAX]

    @property
    def _is_dat(self):
        return isinstance(self._dat, Dat)

    @property
    def _is_INC(self):
        return self._access is INC

    @property
    def _is_MIN(self):
        return self._access is MIN

    @property
    def _is_MAX(self):
        return self._access is MAX

    @property
    def _is_direct(self):
        return isinstance(self._dat, Dat) and self._map is IdentityMap

    @property
    def _is_indirect(self):
        return isinstance(self._dat, Dat) and self._map is not None and self._map is not IdentityMap

    @property
    def _is_indirect_and_not_read(self):
        return self._is_indirect and self._access is not READ

    @property
    def _is_indirect_reduction(self):
        return self._is_indirect and self._access is INC

    @property
    def _uses_itspace(self):
        return self._is_mat or isinstance(self.idx, IterationIndex)


# ------------------------------------------------------------------- HDF5
def _h5_value(slot):
    """The whole content of an HDF5 dataset as a numpy array: ``slot[()]``
    (h5py 2.1 and later), else the ``value`` property the reference uses."""
    try:
        return np.asarray(slot[()])
    except (TypeError, KeyError, IndexError, ValueError):
        return np.asarray(slot.value)


def _h5_str(v):
    return v.decode() if isinstance(v, bytes) else str(v)


# ------------------------------------------------------------------------ Set
class Set(object):
    """OP2 set.  ``size`` is an int or the four sizes core/owned/exec/total."""

    _globalcount = 0

    CORE_SIZE = 0
    OWNED_SIZE = 1
    IMPORT_EXEC_SIZE = 2
    IMPORT_NON_EXEC_SIZE = 3

    @validate_type(('size', (int, np.integer, tuple, list), SizeTypeError),
                   ('name', str, NameTypeError))
    def __init__(self, size=None, dim=1, name=None, halo=None):
        if isinstance(size, (int, np.integer)):
            size = [int(size)] * 4
        size = as_tuple(size, (int, np.integer), 4)
        size = tuple(int(s) for s in size)
        assert size[0] <= size[1] <= size[2] <= size[3], "Set received invalid sizes: %s" % (size,)
        self._core_size, self._size, self._ieh_size, self._inh_size = size
        self._dim = as_tuple(dim, (int, np.integer))
        self._dim = tuple(int(d) for d in self._dim)
        self._cdim = math.prod(self._dim)
        self._name = name or "set_%d" % Set._globalcount
        self._halo = halo
        if self._halo is not None:
            self._halo.verify(self)
        Set._globalcount += 1

    def __call__(self, *dims):
        return IterationSpace(self, dims)

    @classmethod
    def fromhdf5(cls, f, name, dim=1):
        """Construct a Set from the one-element dataset ``name`` of the HDF5
        file ``f`` (an h5py File or an object with its interface); its
        ``dim`` attribute, if present, overrides ``dim``
        (pyop2/base.py:386-394)."""
        slot = f[name]
        if tuple(slot.shape) != (1,):
            raise SizeTypeError("Shape of %s is incorrect" % name)
        size = _h5_value(slot).astype(int)
        dim = slot.attrs.get('dim', dim)
        if isinstance(dim, np.ndarray):
            dim = tuple(int(d) for d in dim.ravel()) if dim.size > 1 else int(dim.ravel()[0])
        elif isinstance(dim, np.integer):
            dim = int(dim)
        return cls(int(size[0]), dim, name)

    @property
    def core_size(self):
        return self._core_size

    @property
    def size(self):
        return self._size

    @property
    def exec_size(self):
        return self._ieh_size

    @property
    def total_size(self):
        return self._inh_size

    @property
    def sizes(self):
        return self._core_size, self._size, self._ieh_size, self._inh_size

    @property
    def dim(self):
        return self._dim

    @property
    def cdim(self):
        return self._cdim

    @property
    def name(self):
        return self._name

    @property
    def halo(self):
        return self._halo

    def __str__(self):
        return "OP2 Set: %s with size %s, dim %s" % (self._name, self._size, self._dim)

    def __repr__(self):
        return "Set(%r, %r, %r)" % (self._size, self._dim, self._name)


class Halo(object):
    """Halo description (pyop2/base.py:402-505): per peer rank, the owned
    elements sent to it and the halo elements received from it.  ``comm`` is
    any communicator of :mod:`pyop2_b200.halo` (a ``torch.distributed`` group,
    in-process ranks) and defaults to the backend's ``MPI.comm``."""

    def __init__(self, sends, receives, comm=None, gnn2unn=None):
        self._sends = tuple(np.asarray(x, dtype=np.int32) for x in sends)
        self._receives = tuple(np.asarray(x, dtype=np.int32) for x in receives)
        self._global_to_petsc_numbering = gnn2unn
        if comm is None:
            comm = _default_comm()
        self._comm = comm
        rank, size = comm.rank, comm.size
        assert len(self._sends) == size, \
            "Invalid number of sends for Halo, got %d, wanted %d" % (len(self._sends), size)
        assert len(self._receives) == size, \
            "Invalid number of receives for Halo, got %d, wanted %d" % (len(self._receives), size)
        assert self._sends[rank].size == 0, "Halo was specified with self-sends on rank %d" % rank
        assert self._receives[rank].size == 0, \
            "Halo was specified with self-receives on rank %d" % rank

    @property
    def comm(self):
        return self._comm

    @property
    def sends(self):
        return self._sends

    @property
    def receives(self):
        return self._receives

    @property
    def global_to_petsc_numbering(self):
        return self._global_to_petsc_numbering

    def verify(self, s):
        for dest, sends in enumerate(self.sends):
            assert (sends >= 0).all() and (sends < s.size).all(), \
                "Halo send to %d is invalid (outside owned elements)" % dest
        for source, receives in enumerate(self.receives):
            assert (receives >= s.size).all() and (receives < s.total_size).all(), \
                "Halo receive from %d is invalid (not in halo elements)" % source


def _default_comm():
    """The selected backend's communicator, else a single rank."""
    mpi = getattr(_BackendSelector._backend, "MPI", None)
    comm = getattr(mpi, "comm", None)
    if comm is None:
        from .halo import SelfComm
        comm = SelfComm()
    return comm


class IterationSpace(object):
    """A Set plus local iteration extents; build it with ``set(e0[, e1])``."""

    @validate_type(('iterset', Set, SetTypeError))
    def __init__(self, iterset, extents=()):
        self._iterset = iterset
        self._extents = as_tuple(extents, (int, np.integer))
        self._extents = tuple(int(e) for e in self._extents)

    @property
    def iterset(self):
        return self._iterset

    @property
    def extents(self):
        return self._extents

    @property
    def name(self):
        return self._iterset.name

    @property
    def core_size(self):
        return self._iterset.core_size

    @property
    def size(self):
        return self._iterset.size

    @property
    def exec_size(self):
        return self._iterset.exec_size

    @property
    def total_size(self):
        return self._iterset.total_size

    def __str__(self):
        return "OP2 Iteration Space: %s with extents %s" % (self._iterset, self._extents)

    def __repr__(self):
        return "IterationSpace(%r, %r)" % (self._iterset, self._extents)


# --------------------------------------------------------------- data carriers
_CTYPES = {"bool": "unsigned char", "int": "int", "int8": "char", "int16": "short",
           "int32": "int", "int64": "long long", "uint8": "unsigned char",
           "uint16": "unsigned short", "uint32": "unsigned int",
           "uint64": "unsigned long long", "float": "double", "float32": "float",
           "float64": "double"}


class DataCarrier(object):
    """Base of Dat (rank 1), Mat (rank 2), Const and Global (rank 0)."""

    @property
    def dtype(self):
        return self._data.dtype

    @property
    def ctype(self):
        return _CTYPES[self.dtype.name]

    @property
    def name(self):
        return self._name

    @property
    def dim(self):
        return self._dim

    @property
    def cdim(self):
        return self._cdim


class Dat(DataCarrier):
    """``dim`` values per element of a :class:`Set`.  Call it with a Map (or
    ``map[idx]``) and an access mode to pass it to a par_loop."""

    _globalcount = 0
    _modes = [READ, WRITE, RW, INC]

    @validate_type(('dataset', Set, SetTypeError), ('name', str, NameTypeError))
    def __init__(self, dataset, data=None, dtype=None, name=None, soa=None, uid=None):
        if data is None:
            try:
                t = np.dtype(dtype) if dtype is not None else np.float64
            except TypeError:
                raise DataTypeError("Invalid data type: %s" % dtype)
            data = np.zeros(dataset.total_size * dataset.cdim, dtype=t)
        self._dataset = dataset
        self._data = verify_reshape(data, dtype, (dataset.total_size,) + dataset.dim,
                                    allow_none=True)
        self._soa = bool(soa)
        self._needs_halo_update = False
        if uid is None:
            self._id = Dat._globalcount
            Dat._globalcount += 1
        else:
            self._id = uid
        self._name = name or "dat_%d" % self._id

    @classmethod
    def fromhdf5(cls, dataset, f, name):
        """Construct a Dat on ``dataset`` from the dataset ``name`` of the
        HDF5 file ``f``; a ``type`` attribute ending in ``:soa`` makes it an
        SoA Dat (pyop2/base.py:842-849)."""
        slot = f[name]
        data = _h5_value(slot)
        soa = _h5_str(slot.attrs['type']).find(':soa') > 0
        return cls(dataset, data, name=name, soa=soa)

    def __call__(self, path, access):
        if access is READ or access is INC or access is WRITE or access is RW:
            return self._arg(path, access)
        return self._call_checked(path, access)

    @validate_in(('access', _modes, ModeValueError))
    def _call_checked(self, path, access):
        return self._arg(path, access)

    def _arg(self, path, access):
        if isinstance(path, Map):
            if path._dataset != self._dataset and path is not IdentityMap:
                raise MapValueError("Dataset of Map does not match Dataset of Dat.")
            return _new_arg(self, path, None, access)
        path._dat = self
        path._access = access
        return path

    @property
    def dataset(self):
        return self._dataset

    @property
    def dim(self):
        return self.dataset.dim

    @property
    def cdim(self):
        return self.dataset.cdim

    @property
    def soa(self):
        return self._soa

    @property
    def data(self):
        if self.dataset.total_size > 0 and self._data.size == 0:
            raise RuntimeError("Illegal access: no data associated with this Dat!")
        maybe_setflags(self._data, write=True)
        self.needs_halo_update = True
        return self._data

    @property
    def data_ro(self):
        if self.dataset.total_size > 0 and self._data.size == 0:
            raise RuntimeError("Illegal access: no data associated with this Dat!")
        maybe_setflags(self._data, write=False)
        return self._data

    @property
    def needs_halo_update(self):
        return self._needs_halo_update

    @needs_halo_update.setter
    def needs_halo_update(self, val):
        self._needs_halo_update = val

    def zero(self):
        """Zero the Dat with a generated direct par_loop (base.py:726-736)."""
        if not hasattr(self, '_zero_kernel'):
            k = """void zero(%(t)s *dat) {
                for (int n = 0; n < %(dim)s; ++n) {
                    dat[n] = (%(t)s)0;
                }
            }""" % {'t': self.ctype, 'dim': self.cdim}
            self._zero_kernel = _make_object('Kernel', k, 'zero')
        _make_object('ParLoop', self._zero_kernel, self.dataset,
                     self(IdentityMap, WRITE)).compute()

    def __str__(self):
        return "OP2 Dat: %s on (%s) with datatype %s" % (self._name, self._dataset, self.dtype.name)

    def __repr__(self):
        return "Dat(%r, '%s', None, '%s')" % (self._dataset, self.dtype, self._name)

    def _check_shape(self, other):
        pass

    def _int_division(self, op):
        """The reference ran under Python 2, where ``/`` between integer
        arrays (the other operand is first cast to this Dat's type,
        pyop2/base.py:749-763) is floor division: an integer Dat divides
        that way, in place too."""
        return (op in (operator.truediv, operator.itruediv)
                and np.issubdtype(self.dtype, np.integer))

    def _op(self, other, op):
        if self._int_division(op):
            op = np.floor_divide
        if np.isscalar(other):
            return _make_object('Dat', self.dataset, op(self.data_ro, as_type(other, self.dtype)),
                                self.dtype)
        self._check_shape(other)
        return _make_object('Dat', self.dataset, op(self.data_ro, as_type(other.data_ro, self.dtype)),
                            self.dtype)

    def _iop(self, other, op):
        if self._int_division(op):
            op = lambda a, b: np.floor_divide(a, b, out=a)   # noqa: E731
        d = self.data
        if np.isscalar(other):
            op(d, as_type(other, self.dtype))
        else:
            self._check_shape(other)
            op(d, as_type(other.data_ro, self.dtype))
        return self

    def __add__(self, other):
        return self._op(other, operator.add)

    def __sub__(self, other):
        return self._op(other, operator.sub)

    def __mul__(self, other):
        return self._op(other, operator.mul)

    def __truediv__(self, other):
        return self._op(other, operator.truediv)

    def __iadd__(self, other):
        return self._iop(other, operator.iadd)

    def __isub__(self, other):
        return self._iop(other, operator.isub)

    def __imul__(self, other):
        return self._iop(other, operator.imul)

    def __itruediv__(self, other):
        return self._iop(other, operator.itruediv)

    @property
    def norm(self):
        """The L2-norm of the flattened values."""
        return np.linalg.norm(self.data_ro)


class Const(DataCarrier):
    """Data constant for every element of every set; globally unique names."""

    class NonUniqueNameError(ValueError):
        """The name of a Const is already in use."""

    _defs = set()
    _globalcount = 0
    _generation = 0     # changes whenever the set of definitions changes

    @validate_type(('name', str, NameTypeError))
    def __init__(self, dim, data=None, name=None, dtype=None):
        self._dim = as_tuple(dim, (int, np.integer))
        self._dim = tuple(int(d) for d in self._dim)
        self._cdim = math.prod(self._dim)
        self._data = verify_reshape(data, dtype, self._dim, allow_none=True)
        self._name = name or "const_%d" % Const._globalcount
        if any(self._name == c._name for c in Const._defs):
            raise Const.NonUniqueNameError(
                "OP2 Constants are globally scoped, %s is already in use" % self._name)
        Const._defs.add(self)
        Const._globalcount += 1
        Const._generation += 1

    @classmethod
    def fromhdf5(cls, f, name):
        """Construct a Const from the dataset ``name`` of the HDF5 file
        ``f``; its shape is the Const's dim (pyop2/base.py:918-926)."""
        slot = f[name]
        dim = tuple(slot.shape)
        data = _h5_value(slot)
        if len(dim) < 1:
            raise DimTypeError("Invalid dimension value %s" % (dim,))
        return cls(dim, data, name)

    @property
    def data(self):
        if len(self._data) == 0:
            raise RuntimeError("Illegal access: No data associated with this Const!")
        return self._data

    @data.setter
    def data(self, value):
        self._data = verify_reshape(value, self.dtype, self.dim)

    def __str__(self):
        return "OP2 Const: %s of dim %s and type %s with value %s" % \
            (self._name, self._dim, self._data.dtype.name, self._data)

    def __repr__(self):
        return "Const(%s, %s, '%s')" % (self._dim, self._data, self._name)

    @classmethod
    def _definitions(cls):
        return sorted(Const._defs, key=lambda c: c.name)

    def remove_from_namespace(self):
        """Remove this Const from the namespace (the name may be reused)."""
        Const._defs.discard(self)
        Const._generation += 1

    def _format_declaration(self):
        d = {'type': self.ctype, 'name': self.name, 'dim': self.cdim}
        if self.cdim == 1:
            return "static %(type)s %(name)s;" % d
        return "static %(type)s %(name)s[%(dim)s];" % d


class Global(DataCarrier):
    """A global value: READ, or reduced with INC/MIN/MAX over a par_loop."""

    _globalcount = 0
    _modes = [READ, INC, MIN, MAX]

    @validate_type(('name', str, NameTypeError))
    def __init__(self, dim, data=None, dtype=None, name=None):
        if type(dim) is int:
            # the usual scalar Global of a reduction (a fresh one per loop
            # call in the demos): no tuple normalisation
            self._dim = (dim,)
        else:
            self._dim = tuple(int(d) for d in as_tuple(dim, (int, np.integer)))
        self._cdim = math.prod(self._dim)
        self._data = verify_reshape(data, dtype, self._dim, allow_none=True)
        self._name = name or "global_%d" % Global._globalcount
        Global._globalcount += 1

    @validate_in(('access', _modes, ModeValueError))
    def __call__(self, access):
        return _new_arg(self, None, None, access)

    def __str__(self):
        return "OP2 Global Argument: %s with dim %s and value %s" % (self._name, self._dim, self._data)

    def __repr__(self):
        return "Global('%s', %r, %r)" % (self._name, self._dim, self._data)

    @property
    def data(self):
        if len(self._data) == 0:
            raise RuntimeError("Illegal access: No data associated with this Global!")
        return self._data

    @data.setter
    def data(self, value):
        self._data = verify_reshape(value, self.dtype, self.dim)

    @property
    def soa(self):
        return False


# ------------------------------------------------------------ iteration index
class IterationIndex(object):
    """Iteration-space index; use ``op2.i[n]``."""

    def __init__(self, index=None):
        assert index is None or isinstance(index, int), "i must be an int"
        self._index = index

    def __str__(self):
        return "OP2 IterationIndex: %s" % self._index

    def __repr__(self):
        return "IterationIndex(%r)" % self._index

    @property
    def index(self):
        return self._index

    def __getitem__(self, idx):
        return IterationIndex(idx)

    def __iter__(self):
        yield self


i = IterationIndex()


# ------------------------------------------------------------------------ Map
class Map(object):
    """Fixed-arity int32 connectivity from ``iterset`` to ``dataset``."""

    _globalcount = 0

    @validate_type(('iterset', Set, SetTypeError), ('dataset', Set, SetTypeError),
                   ('dim', (int, np.integer), DimTypeError), ('name', str, NameTypeError))
    def __init__(self, iterset, dataset, dim, values=None, name=None):
        self._iterset = iterset
        self._dataset = dataset
        self._dim = int(dim)
        self._values = verify_reshape(values, np.int32, (iterset.total_size, self._dim),
                                      allow_none=True)
        self._name = name or "map_%d" % Map._globalcount
        Map._globalcount += 1

    @classmethod
    def fromhdf5(cls, iterset, dataset, f, name):
        """Construct a Map from ``iterset`` to ``dataset`` from the
        two-dimensional dataset ``name`` of the HDF5 file ``f`` (its second
        extent is the arity; pyop2/base.py:1117-1125)."""
        slot = f[name]
        values = _h5_value(slot)
        dim = tuple(slot.shape)[1:]
        if len(dim) != 1:
            raise DimTypeError("Unrecognised dimension value %s" % (dim,))
        return cls(iterset, dataset, dim[0], values, name)

    def __getitem__(self, index):
        # the common case first: a Python int within the arity
        if type(index) is int and 0 <= index < self._dim:
            return _new_arg(None, self, index, None)
        if isinstance(index, slice):
            # test/unit/test_api.py:655-660: slicing a Map is not supported
            raise NotImplementedError("Slicing maps is not allowed")
        return self._getitem_checked(index)

    @validate_type(('index', (int, np.integer, IterationIndex), IndexTypeError))
    def _getitem_checked(self, index):
        if isinstance(index, (int, np.integer)) and not (0 <= index < self._dim):
            raise IndexValueError("Index must be in interval [0,%d]" % (self._dim - 1))
        if isinstance(index, IterationIndex) and index.index not in [0, 1]:
            raise IndexValueError("IterationIndex must be in interval [0,1]")
        if isinstance(index, np.integer):
            index = int(index)
        return _make_object('Arg', map=self, idx=index)

    def __iter__(self):
        yield self

    @property
    def iterset(self):
        return self._iterset

    @property
    def dataset(self):
        return self._dataset

    @property
    def dim(self):
        return self._dim

    @property
    def values(self):
        return self._values

    @property
    def name(self):
        return self._name

    def __str__(self):
        return "OP2 Map: %s from (%s) to (%s) with dim %s" % \
            (self._name, self._iterset, self._dataset, self._dim)

    def __repr__(self):
        return "Map(%r, %r, %s, None, '%s')" % (self._iterset, self._dataset, self._dim, self._name)

    def __eq__(self, o):
        try:
            return (self._iterset == o._iterset and self._dataset == o._dataset and
                    self._dim == o.dim and self._name == o.name)
        except AttributeError:
            return False

    def __ne__(self, o):
        return not self.__eq__(o)

    def __hash__(self):
        return id(self)


IdentityMap = Map(Set(0), Set(0), 1, [], 'identity')


# ------------------------------------------------------------------- Sparsity
class Sparsity(Cached):
    """CSR pattern from the union of outer products of (row, col) Map pairs.

    ``Sparsity(map)``, ``Sparsity((rmap, cmap))`` or
    ``Sparsity(((rmap0, cmap0), (rmap1, cmap1)))``."""

    _cache = {}
    _globalcount = 0

    @classmethod
    @validate_type(('maps', (Map, tuple), MapTypeError),)
    def _process_args(cls, maps, name=None, *args, **kwargs):
        assert not name or isinstance(name, str), "Name must be of type str"
        maps = (maps, maps) if isinstance(maps, Map) else maps
        maps = (maps,) if isinstance(maps[0], Map) else maps
        for pair in maps:
            for m in pair:
                if not isinstance(m, Map):
                    raise MapTypeError("All maps must be of type map, not type %r" % type(m))
                if len(m.values) == 0:
                    raise MapValueError("Unpopulated map values when trying to build sparsity.")
        # canonical order of the pairs (the reference sorted them by object order)
        maps = tuple(sorted((tuple(p) for p in maps), key=lambda p: (id(p[0]), id(p[1]))))
        return [maps, name], {}

    @classmethod
    def _cache_key(cls, maps, *args, **kwargs):
        return maps

    def __init__(self, maps, name=None):
        if self._initialized:
            return
        self._rmaps, self._cmaps = zip(*maps)
        assert len(self._rmaps) == len(self._cmaps), "Must pass equal number of row and column maps"
        for pair in maps:
            if pair[0].iterset is not pair[1].iterset:
                raise RuntimeError("Iterset of both maps in a pair must be the same")
        if not all(m.dataset is self._rmaps[0].dataset for m in self._rmaps):
            raise RuntimeError("Dataset of all row maps must be the same")
        if not all(m.dataset is self._cmaps[0].dataset for m in self._cmaps):
            raise RuntimeError("Dataset of all column maps must be the same")
        self._nrows = self._rmaps[0].dataset.size
        self._ncols = self._cmaps[0].dataset.size
        self._dims = (self._rmaps[0].dataset.cdim, self._cmaps[0].dataset.cdim)
        self._name = name or "sparsity_%d" % Sparsity._globalcount
        Sparsity._globalcount += 1
        self._build()
        self._initialized = True

    def _build(self):
        raise NotImplementedError("Sparsity construction is provided by the backend")

    @property
    def _nmaps(self):
        return len(self._rmaps)

    @property
    def maps(self):
        return list(zip(self._rmaps, self._cmaps))

    @property
    def cmaps(self):
        return self._cmaps

    @property
    def rmaps(self):
        return self._rmaps

    @property
    def dims(self):
        return self._dims

    @property
    def nrows(self):
        return self._nrows

    @property
    def ncols(self):
        return self._ncols

    @property
    def name(self):
        return self._name

    def __str__(self):
        return "OP2 Sparsity: rmaps %s, cmaps %s, name %s" % (self._rmaps, self._cmaps, self._name)

    def __repr__(self):
        return "Sparsity(%r, %r)" % (tuple(self.maps), self.name)

    @property
    def rowptr(self):
        return self._rowptr

    @property
    def colidx(self):
        return self._colidx

    @property
    def nnz(self):
        return self._d_nnz

    @property
    def onnz(self):
        return self._o_nnz

    @property
    def nz(self):
        return int(self._d_nz)

    @property
    def onz(self):
        return int(self._o_nz)


# ------------------------------------------------------------------------ Mat
class Mat(DataCarrier):
    """Values on a :class:`Sparsity`; call with ``(rmap[i[0]], cmap[i[1]])``."""

    _globalcount = 0
    _modes = [WRITE, INC]

    @validate_type(('sparsity', Sparsity, SparsityTypeError), ('name', str, NameTypeError))
    def __init__(self, sparsity, dtype=None, name=None):
        self._sparsity = sparsity
        self._datatype = np.dtype(dtype)
        self._name = name or "mat_%d" % Mat._globalcount
        Mat._globalcount += 1

    @validate_in(('access', _modes, ModeValueError))
    def __call__(self, path, access):
        path = as_tuple(path, Arg, 2)
        path_maps = [arg.map for arg in path]
        path_idxs = [arg.idx for arg in path]
        if not any(path_maps[0] == p[0] and path_maps[1] == p[1] for p in self.sparsity.maps):
            raise MapValueError("Path maps not in sparsity maps")
        return _make_object('Arg', data=self, map=path_maps, access=access, idx=path_idxs)

    @property
    def dims(self):
        return self._sparsity._dims

    @property
    def sparsity(self):
        return self._sparsity

    @property
    def _is_scalar_field(self):
        return np.prod(self.dims) == 1

    @property
    def _is_vector_field(self):
        return not self._is_scalar_field

    @property
    def values(self):
        raise NotImplementedError("Abstract base Mat does not implement values()")

    @property
    def dtype(self):
        return self._datatype

    def __str__(self):
        return "OP2 Mat: %s, sparsity (%s), datatype %s" % (self._name, self._sparsity, self._datatype.name)

    def __repr__(self):
        return "Mat(%r, '%s', '%s')" % (self._sparsity, self._datatype, self._name)


# --------------------------------------------------------------------- Kernel
class Kernel(Cached):
    """A C function processing ONE element of the iteration set."""

    _globalcount = 0
    _cache = {}

    @classmethod
    @validate_type(('name', str, NameTypeError))
    def _cache_key(cls, code, name):
        return md5((code + name).encode()).hexdigest()

    def __init__(self, code, name):
        if self._initialized:
            return
        self._name = name or "kernel_%d" % Kernel._globalcount
        self._code = code
        Kernel._globalcount += 1
        self._initialized = True

    @property
    def name(self):
        return self._name

    @property
    def code(self):
        return self._code

    def __str__(self):
        return "OP2 Kernel: %s" % self._name

    def __repr__(self):
        return 'Kernel("""%s""", "%s")' % (self._code, self._name)


class JITModule(Cached):
    """Cached compiled par_loop stub; the key is pyop2/base.py:1444-1471's."""

    _cache = {}

    @classmethod
    def _cache_key(cls, kernel, itspace_extents, *args, **kwargs):
        key = (kernel.cache_key, itspace_extents)
        for arg in args:
            if arg._is_global:
                key += (arg.data.dim, arg.data.dtype, arg.access)
            elif arg._is_dat:
                if isinstance(arg.idx, IterationIndex):
                    idx = (arg.idx.__class__, arg.idx.index)
                else:
                    idx = arg.idx
                map_dim = None if arg.map is IdentityMap else arg.map.dim
                key += (arg.data.dim, arg.data.dtype, map_dim, idx, arg.access, arg.data.soa)
            elif arg._is_mat:
                idxs = (arg.idx[0].__class__, arg.idx[0].index, arg.idx[1].index)
                map_dims = (arg.map[0].dim, arg.map[1].dim)
                key += (arg.data.dims, arg.data.dtype, idxs, map_dims, arg.access)
        for c in Const._definitions():
            key += (c.name, c.dtype, c.cdim)
        return key


# -------------------------------------------------------------------- ParLoop
class ParLoop(object):
    """Kernel, iteration space and arguments of one parallel loop."""

    def __init__(self, kernel, itspace, *args):
        self._actual_args = args
        self._kernel = kernel
        self._it_space = itspace if isinstance(itspace, IterationSpace) else IterationSpace(itspace)
        self.check_args()

    def compute(self):
        raise RuntimeError('Must select a backend')

    def maybe_set_halo_update_needed(self):
        for arg in self.args:
            if arg._is_dat and arg.access in [INC, WRITE, RW]:
                arg.data.needs_halo_update = True

    def check_args(self):
        """Iteration set of every map must be the loop's; the dataset of every
        Dat's map must be the Dat's set (MapValueError otherwise)."""
        iterset = self._it_space._iterset
        for i, arg in enumerate(self._actual_args):
            if arg._is_global or arg._map is IdentityMap:
                continue
            for j, m in enumerate(as_tuple(arg._map)):
                if m._iterset != iterset:
                    raise MapValueError("Iterset of arg %s map %s doesn't match ParLoop iterset." % (i, j))
                if arg._is_mat:
                    continue
                if m._dataset != arg.data._dataset:
                    raise MapValueError("Dataset of arg %s map %s doesn't match the set of its Dat." % (i, j))

    @property
    def it_space(self):
        return self._it_space

    @property
    def is_direct(self):
        return all(a.map is None or a.map is IdentityMap for a in self.args)

    @property
    def is_indirect(self):
        return not self.is_direct

    @property
    def needs_exec_halo(self):
        return any(arg._is_indirect_and_not_read or arg._is_mat for arg in self.args)

    @property
    def kernel(self):
        return self._kernel

    @property
    def args(self):
        return self._actual_args

    @property
    def _has_soa(self):
        return any(a._is_soa for a in self._actual_args)


DEFAULT_SOLVER_PARAMETERS = {'linear_solver': 'cg',
                             'preconditioner': 'jacobi',
                             'relative_tolerance': 1.0e-7,
                             'absolute_tolerance': 1.0e-50,
                             'divergence_tolerance': 1.0e+4,
                             'maximum_iterations': 1000,
                             'monitor_convergence': False,
                             'plot_convergence': False,
                             'plot_prefix': '',
                             'error_on_nonconvergence': True,
                             'gmres_restart': 30}


class Solver(object):
    """Linear solver parameters (pyop2/base.py:1607-1657)."""

    def __init__(self, parameters=None, **kwargs):
        self.parameters = DEFAULT_SOLVER_PARAMETERS.copy()
        if parameters and kwargs:
            raise RuntimeError("Solver options are set either by parameters or kwargs")
        if parameters:
            self.parameters.update(parameters)
        else:
            self.parameters.update(kwargs)

    def update_parameters(self, parameters):
        self.parameters.update(parameters)

    def solve(self, A, x, b):
        raise NotImplementedError("solve must be implemented by backend")
