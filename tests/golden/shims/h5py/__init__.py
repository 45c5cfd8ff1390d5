"""In-memory stand-in for the subset of h5py the reference uses (test infrastructure).

Files live in a process-wide registry keyed by absolute path; an empty marker
file is written on disk so ``os.path.isfile`` checks in the reference pass and
``shutil.copy`` of an MPS file works.  Datasets expose ``.value``, ``.shape``,
``.attrs`` and NumPy indexing; groups support create_group, item assignment,
``in``, iteration, deletion and nested "a/b" paths.
"""
import os
import numpy

_REGISTRY = {}


class Dataset(object):
    def __init__(self, data):
        self._data = numpy.array(data)
        self.attrs = {}

    @property
    def value(self):
        # as h5py: a scalar dataset reads as a NumPy scalar, an array dataset as an array
        return self._data[()] if self._data.ndim == 0 else self._data.copy()

    @property
    def shape(self):
        return self._data.shape

    @property
    def dtype(self):
        return self._data.dtype

    def __getitem__(self, idx):
        return self._data[idx]

    def __len__(self):
        return len(self._data)


class Group(object):
    def __init__(self):
        self._items = {}
        self.attrs = {}

    def _walk(self, name, create=False):
        parts = [p for p in name.split("/") if p]
        g = self
        for p in parts[:-1]:
            if p not in g._items:
                if not create:
                    raise KeyError(name)
                g._items[p] = Group()
            g = g._items[p]
        return g, parts[-1]

    def create_group(self, name):
        g, last = self._walk(name, create=True)
        if last in g._items:
            raise ValueError("exists: " + name)
        ng = Group()
        g._items[last] = ng
        return ng

    def create_dataset(self, name, shape=None, dtype=None, data=None, **kw):
        if data is None:
            data = numpy.zeros(shape, dtype=dtype)
        g, last = self._walk(name, create=True)
        ds = Dataset(data)
        g._items[last] = ds
        return ds

    def __setitem__(self, name, data):
        g, last = self._walk(name, create=True)
        g._items[last] = Dataset(data)

    def __getitem__(self, name):
        g, last = self._walk(name)
        return g._items[last]

    def __contains__(self, name):
        try:
            g, last = self._walk(name)
        except KeyError:
            return False
        return last in g._items

    def __delitem__(self, name):
        g, last = self._walk(name)
        del g._items[last]

    def __iter__(self):
        return iter(list(self._items.keys()))

    def keys(self):
        return list(self._items.keys())


class File(Group):
    def __init__(self, name, mode="a", **kw):
        path = os.path.abspath(name)
        self.filename = path
        if mode == "w" or (mode in ("a", "w-", "x") and path not in _REGISTRY):
            root = Group()
            _REGISTRY[path] = root
            with open(path, "w") as f:
                f.write("h5py-shim\n")
        else:
            if path not in _REGISTRY:
                # a copy made by shutil.copy of a marker file: share nothing
                raise IOError("Unable to open file (shim): " + path)
            root = _REGISTRY[path]
        self._items = root._items
        self.attrs = root.attrs

    def close(self):
        pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
