"""In-memory stand-in for ``h5py`` so ipie's driver runs without HDF5.

ipie's estimator handler writes block data with ``h5py.File(name, mode)``
used as a context manager and dataset assignment by path.  This shim keeps
every "file" as a dict of numpy arrays in ``FILES`` so the fixture script can
read the block estimates back.  Only ``tests/golden/make_golden.py`` uses it.
"""
import numpy as _np

FILES = {}


class File:
    def __init__(self, name, mode="r", **kwargs):
        if mode == "w" or name not in FILES:
            FILES[name] = {}
        self._d = FILES[name]

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def close(self):
        pass

    def __setitem__(self, key, value):
        self._d[key] = _np.array(value)

    def __getitem__(self, key):
        return self._d[key]

    def __contains__(self, key):
        return key in self._d

    def keys(self):
        return self._d.keys()
