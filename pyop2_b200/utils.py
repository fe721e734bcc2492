"""Common utilities of the OP2 host layer.

Behaviour follows pyop2/utils.py: ``as_tuple`` (:48-63), ``as_type`` (:65-77),
the argument validation decorators (:79-162), ``verify_reshape`` (:164-187),
``align`` (:189-191), ``uniquify`` (:193-196), the argparse ``parser``
(:198-224) and ``maybe_setflags`` (:226-232).
"""

import argparse
import functools

import numpy as np

from .exceptions import DataTypeError, DataValueError


def as_tuple(item, type=None, length=None):
    if item is None:
        t = []
    else:
        try:
            t = tuple(item)
        except TypeError:
            t = (item,) * (length or 1)
    if length and not len(t) == length:
        raise ValueError("Tuple needs to be of length %d" % length)
    if type and not all(isinstance(i, type) for i in t):
        raise TypeError("Items need to be of type %s" % type)
    return t


def as_type(obj, typ):
    """Return obj if it is of dtype typ, otherwise a copy cast to typ."""
    try:
        return obj if obj.dtype == typ else obj.astype(typ)
    except AttributeError:
        if isinstance(obj, int):
            return np.int64(obj).astype(typ)
        elif isinstance(obj, float):
            return np.float64(obj).astype(typ)
        raise TypeError("Invalid type %s" % type(obj))


class _validate_base(object):
    """Decorator validating named arguments of the decorated function.

    Formal parameters absent from the function and actual arguments that are
    not passed are ignored; an argument equal to its default is accepted."""

    def __init__(self, *checks):
        self._checks = checks

    def __call__(self, f):
        code = f.__code__
        varnames = code.co_varnames[:code.co_argcount]
        defaults = f.__defaults__ or ()
        where = "%s:%d" % (code.co_filename, code.co_firstlineno + 1)
        # positions resolved once: (name, position, index into defaults or -1)
        plan = []
        for argname, cond, exception in self._checks:
            if argname in varnames:
                i = varnames.index(argname)
                di = i - len(varnames) + len(defaults)
                plan.append((argname, i, di, cond, exception))
        check = self.check_arg

        @functools.wraps(f)
        def wrapper(*args, **kwargs):
            n = len(args)
            for argname, i, di, cond, exception in plan:
                if i < n:
                    arg = args[i]
                elif kwargs and argname in kwargs:
                    arg = kwargs[argname]
                else:
                    continue
                if di >= 0:
                    d = defaults[di]
                    if arg is d:
                        continue
                    try:
                        if not isinstance(arg, np.ndarray) and arg == d:
                            continue
                    except Exception:
                        pass
                check(arg, cond, exception, where)
            return f(*args, **kwargs)
        return wrapper


class validate_type(_validate_base):
    """Validate argument types: checks are (name, type, exception)."""

    def check_arg(self, arg, argtype, exception, where):
        if not isinstance(arg, argtype):
            raise exception("%s Parameter %s must be of type %r" % (where, arg, argtype))


class validate_in(_validate_base):
    """Validate arguments are in a list: checks are (name, list, exception)."""

    def check_arg(self, arg, values, exception, where):
        if not any(arg is v for v in values) and arg not in values:
            raise exception("%s %s must be one of %s" % (where, arg, values))


class validate_range(_validate_base):
    """Validate numeric range: checks are (name, (lo, hi), exception)."""

    def check_arg(self, arg, range, exception, where):
        if not range[0] <= arg <= range[1]:
            raise exception("%s %s must be within range %s" % (where, arg, range))


def verify_reshape(data, dtype, shape, allow_none=False):
    """Verify data is of type dtype and try to reshape it to shape."""
    try:
        t = np.dtype(dtype) if dtype is not None else None
    except TypeError:
        raise DataTypeError("Invalid data type: %s" % dtype)
    if data is None and allow_none:
        return np.asarray([], dtype=t)
    elif data is None:
        raise DataValueError("Invalid data: None is not allowed!")
    if isinstance(data, (int, float)) and shape in ((1,), 1):
        # a scalar (a Global's or Const's usual value): no array round trip
        return np.array([data], dtype=t if t is not None else np.asarray(data).dtype)
    try:
        a = np.asarray(data, dtype=t)
    except (ValueError, TypeError):
        raise DataValueError("Invalid data: cannot convert to %s!" % dtype)
    try:
        # Reshape in place like the reference (pyop2/utils.py:180-184), so the
        # array keeps owning its data; a non-contiguous input is copied first.
        if not a.flags['C_CONTIGUOUS']:
            a = np.ascontiguousarray(a)
        a.shape = shape
        return a
    except (ValueError, AttributeError):
        raise DataValueError("Invalid data: expected %d values, got %d!" %
                             (np.prod(shape), np.asarray(data).size))


def align(nbytes, alignment=16):
    """Round nbytes up to a multiple of alignment."""
    return ((nbytes + alignment - 1) // alignment) * alignment


def uniquify(iterable):
    """Remove duplicates but preserve order."""
    seen = set()
    return [x for x in iterable if x not in seen and (seen.add(x) or True)]


def parser(description=None, group=False):
    """argparse parser with the OP2 backend options."""
    p = argparse.ArgumentParser(description=description, add_help=True, prefix_chars="-",
                                formatter_class=argparse.RawDescriptionHelpFormatter)
    g = p.add_argument_group('pyop2', 'backend configuration options') if group else p
    g.add_argument('-b', '--backend', default='b200', choices=['b200'],
                   help='select pyop2 backend')
    g.add_argument('-d', '--debug', default=argparse.SUPPRESS, type=int, choices=range(8),
                   help='set pyop2 debug level')
    g.add_argument('-l', '--log-level', default='WARN',
                   choices=['CRITICAL', 'ERROR', 'WARN', 'INFO', 'DEBUG'],
                   help='set pyop2 logging level (default=WARN)')
    return p


def parse_args(*args, **kwargs):
    return vars(parser(*args, **kwargs).parse_args())


def maybe_setflags(array, write=None, align=None, uic=None):
    """Set flags on a numpy array, but only the write flag of arrays owning
    their data (numpy refuses it otherwise)."""
    write = write if array.flags['OWNDATA'] else None
    array.setflags(write=write, align=align, uic=uic)
