"""Keyed object cache (pyop2/caching.py:41-96).

``Cached.__new__`` computes a key from the processed constructor arguments and
returns the cached instance when one exists; otherwise it builds, stores and
returns a new one.  A key of None disables caching for that call.
"""


class Cached(object):

    def __new__(cls, *args, **kwargs):
        args, kwargs = cls._process_args(*args, **kwargs)
        key = cls._cache_key(*args, **kwargs)
        try:
            return cls._cache_lookup(key)
        except (KeyError, TypeError):
            obj = super(Cached, cls).__new__(cls)
            obj._key = key
            obj._initialized = False
            obj.__init__(*args, **kwargs)
            if key is not None:
                cls._cache_store(key, obj)
            return obj

    @classmethod
    def _cache_lookup(cls, key):
        return cls._cache[key]

    @classmethod
    def _cache_store(cls, key, val):
        cls._cache[key] = val

    @classmethod
    def _process_args(cls, *args, **kwargs):
        return args, kwargs

    @classmethod
    def _cache_key(cls, *args, **kwargs):
        return tuple(args) + tuple(sorted(kwargs.items()))

    @property
    def cache_key(self):
        return self._key
