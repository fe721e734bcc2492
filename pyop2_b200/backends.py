"""Backend selection (pyop2/backends.py:44-150).

The ``op2`` classes use :class:`_BackendSelector` as metaclass: constructing
``op2.Dat(...)`` instantiates the class of the same name in the selected
backend module.  Backends are modules ``pyop2_b200.<name>``; ``b200`` is the
CUDA backend.  Before ``op2.init`` the selector points at a placeholder whose
constructors raise, and after ``op2.exit`` at one that refuses re-use.
"""

import importlib
import types

from .logger import warning


def _placeholder(modname, message):
    mod = types.ModuleType(modname)

    def _fail(*args, **kwargs):
        raise RuntimeError(message)

    for name in ("Kernel", "Set", "Halo", "Dat", "Mat", "Const", "Global", "Map", "Sparsity",
                 "Solver", "IterationSpace", "ParLoop", "Arg"):
        setattr(mod, name, _fail)
    mod.par_loop = _fail
    mod._setup = lambda: None
    return mod


void = _placeholder("pyop2_b200.void", "Must select a backend: call op2.init() first")
finalised = _placeholder("pyop2_b200.finalised", "op2.exit has been called")

backends = {'void': void, 'finalised': finalised}


def _make_object(obj, *args, **kwargs):
    """Instantiate class ``obj`` of the selected backend."""
    try:
        t = _BackendSelector._backend.__dict__[obj]
    except KeyError:
        warning('Backend %s does not appear to implement class %s'
                % (_BackendSelector._backend.__name__, obj))
        raise
    return t(*args, **kwargs)


class _BackendSelector(type):
    """Metaclass: instantiating a class makes an object of the backend's class
    of the same name."""

    _backend = void

    def __new__(mcs, name, bases, dct):
        if not dct.get('__doc__'):
            for b in bases:
                for c in b.mro():
                    if c.__doc__:
                        dct['__doc__'] = c.__doc__
                        break
                if dct.get('__doc__'):
                    break
        return type.__new__(mcs, name, bases, dct)

    def __call__(cls, *args, **kwargs):
        try:
            t = cls._backend.__dict__[cls.__name__]
        except KeyError:
            warning('Backend %s does not appear to implement class %s'
                    % (cls._backend.__name__, cls.__name__))
            raise
        return t(*args, **kwargs)


def get_backend():
    return _BackendSelector._backend.__name__


def set_backend(backend):
    if _BackendSelector._backend is not void:
        raise RuntimeError("The backend can only be set once!")
    mod = backends.get(backend)
    if mod is None:
        try:
            mod = importlib.import_module('pyop2_b200.%s' % backend)
        except ImportError:
            warning('Unable to import backend %s' % backend)
            raise
    backends[backend] = mod
    _BackendSelector._backend = mod


def unset_backend():
    _BackendSelector._backend = finalised


def reset_backend():
    """Return to the uninitialised state (used between test sessions)."""
    _BackendSelector._backend = void
