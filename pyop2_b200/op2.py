"""The OP2 API (pyop2/op2.py:49-164): ``init``/``exit``, the data classes,
``par_loop`` and ``solve``.  ``op2.init(backend='b200')`` selects the B200
CUDA backend (the default)."""

import atexit

from . import backends, base
from . import configuration as cfg
from .base import READ, WRITE, RW, INC, MIN, MAX, IdentityMap, i  # noqa: F401
from .exceptions import DatTypeError, MatTypeError
from .logger import critical, debug, error, info, set_log_level, warning  # noqa: F401
from .utils import validate_type


def init(**kwargs):
    """Initialise OP2: select the backend and set configuration options.

    :arg backend: the backend, ``"b200"``.
    :arg debug: debug level.
    Further keys: see :mod:`pyop2_b200.configuration`.

    Calling ``init`` again with another backend, or after ``exit``, raises
    RuntimeError; calling it again with the same backend updates the
    configuration."""
    comm = kwargs.pop('comm', None)
    backend = backends.get_backend()
    if backend == 'pyop2_b200.finalised':
        raise RuntimeError("Calling init() after exit() is illegal.")
    if 'backend' in kwargs and backend not in ('pyop2_b200.void', 'pyop2_b200.' + kwargs['backend']):
        raise RuntimeError("Changing the backend is not possible once set.")
    cfg.configure(**kwargs)
    set_log_level(cfg.cfg['log_level'])
    if backend == 'pyop2_b200.void':
        backends.set_backend(cfg.cfg['backend'])
        try:
            backends._BackendSelector._backend._setup()
        except Exception:
            backends.reset_backend()
            raise
    else:
        # the backend may have been selected without a device (host-only
        # use of the data classes); setting up is idempotent
        backends._BackendSelector._backend._setup()
    if comm is not None:
        # pyop2/op2.py:78-79: the communicator of partitioned runs
        backends._BackendSelector._backend.MPI.comm = comm
    global MPI
    MPI = backends._BackendSelector._backend.MPI


@atexit.register
def exit():
    """Exit OP2 and release the backend."""
    cfg.reset()
    if backends.get_backend() not in ('pyop2_b200.void', 'pyop2_b200.finalised'):
        mod = backends._BackendSelector._backend
        if hasattr(mod, '_teardown'):
            mod._teardown()
        backends.unset_backend()


class IterationSpace(base.IterationSpace, metaclass=backends._BackendSelector):
    pass


class Kernel(base.Kernel, metaclass=backends._BackendSelector):
    pass


class Set(base.Set, metaclass=backends._BackendSelector):
    pass


class Halo(base.Halo, metaclass=backends._BackendSelector):
    pass


class Dat(base.Dat, metaclass=backends._BackendSelector):
    pass


class Mat(base.Mat, metaclass=backends._BackendSelector):
    pass


class Const(base.Const, metaclass=backends._BackendSelector):
    NonUniqueNameError = base.Const.NonUniqueNameError


class Global(base.Global, metaclass=backends._BackendSelector):
    pass


class Map(base.Map, metaclass=backends._BackendSelector):
    pass


class Sparsity(base.Sparsity, metaclass=backends._BackendSelector):
    pass


class Solver(base.Solver, metaclass=backends._BackendSelector):
    pass


class _SingleRank(object):
    """Single-process communicator stand-in (MPI is not used on one GPU)."""
    rank = 0
    size = 1


class _MPIConfig(object):
    comm = _SingleRank()
    parallel = False


MPI = _MPIConfig()


def par_loop(kernel, it_space, *args):
    """Run ``kernel`` over every element of ``it_space`` (a Set, or a Set with
    local extents ``set(e0[, e1])``) with the given Dat/Mat/Global args."""
    return backends._BackendSelector._backend.par_loop(kernel, it_space, *args)


@validate_type(('M', base.Mat, MatTypeError), ('x', base.Dat, DatTypeError),
               ('b', base.Dat, DatTypeError))
def solve(M, x, b):
    """Solve M x = b with the default Solver parameters."""
    Solver().solve(M, x, b)
