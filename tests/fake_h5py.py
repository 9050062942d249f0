"""A dict-backed stand-in for the part of ``h5py`` the self-energy cache uses.

TEST INFRASTRUCTURE ONLY.  h5py is not installed in this image; the reference's
``write_to_hdf5`` / ``read_from_hdf5`` / ``merge_hdf5_files``
(negf/lead_property.py:932-984) and the mirrors in ``dpnegf_b200.lead_property``
only call ``h5py.File(path, mode)`` as a context manager, ``require_group``,
``create_dataset(name, data=..., compression=...)``, ``flush``, ``in``, item
access, iteration and ``Group.copy``, and read a dataset with ``[:]``.  This
module provides exactly those, keeping every "file" in memory keyed by its path,
so a file written through one implementation can be read through the other.
"""
import types

import numpy as np

FILES = {}


class Dataset:
    def __init__(self, data):
        self.data = np.array(data, copy=True)

    def __getitem__(self, key):
        return self.data[key]


class Group(dict):
    def require_group(self, name):
        g = self.get(name)
        if g is None:
            g = self[name] = Group()
        if not isinstance(g, Group):
            raise TypeError(f"{name} is not a group")
        return g

    def create_dataset(self, name, data=None, compression=None, **kw):
        if name in self:
            raise ValueError(f"Unable to create dataset (name already exists): {name}")
        self[name] = Dataset(data)
        return self[name]

    def copy(self, name, dest):
        dest[name] = Dataset(self[name].data)


class File(Group):
    def __init__(self, path, mode="r"):
        super().__init__()
        self._path = str(path)
        if mode == "r" and self._path not in FILES:
            raise FileNotFoundError(f"Unable to open file (file does not exist): {path}")
        if mode == "w":
            FILES[self._path] = Group()
        self.update(FILES.setdefault(self._path, Group()))

    def flush(self):
        FILES[self._path] = Group(self)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.flush()
        return False


def module():
    """A module object to put in ``sys.modules["h5py"]``."""
    m = types.ModuleType("h5py")
    m.File = File
    return m


def keys(path):
    """{group: {dataset: ndarray}} of an in-memory file."""
    return {g: {d: ds.data for d, ds in grp.items()} for g, grp in FILES.get(str(path), {}).items()}
