"""An in-memory stand-in for the part of the h5py API the archive codec uses
(``File`` with modes "r", "r+", "w"; groups with ``attrs``, ``create_group``,
``create_dataset``, ``keys``, membership and indexing; datasets with ``[()]``,
``[...] = v``, ``dtype``, ``compression``, ``compression_opts``, ``chunks``). h5py is
not installed in this image; the stand-in keeps each file as a pickle on disk so
paths behave like files. Attribute values come back as h5py returns them: text as
``str``, integers as numpy integers."""

import pickle
from pathlib import Path

import numpy as np


class _Attrs(dict):
    def __setitem__(self, key, value):
        if isinstance(value, (bool, np.bool_)):
            value = np.bool_(value)
        elif isinstance(value, (int, np.integer)):
            value = np.int64(value)
        elif isinstance(value, float):
            value = np.float64(value)
        super().__setitem__(key, value)


class Dataset:
    def __init__(self, data, compression=None, compression_opts=None, shuffle=False):
        self._data = np.array(data, copy=True)
        self.compression = compression
        self.compression_opts = compression_opts
        self.shuffle = shuffle
        self.chunks = tuple(min(64, d) for d in self._data.shape) if compression else None
        self.attrs = _Attrs()

    @property
    def dtype(self):
        return self._data.dtype

    def __getitem__(self, key):
        return self._data[key].copy() if isinstance(self._data[key], np.ndarray) else self._data[key]

    def __setitem__(self, key, value):
        self._data[key] = value


class Group:
    def __init__(self):
        self.attrs = _Attrs()
        self._children = {}

    def create_group(self, name):
        if name in self._children:
            raise ValueError(f"name already exists: {name}")
        g = Group()
        self._children[name] = g
        return g

    def create_dataset(self, name, data=None, **options):
        if name in self._children:
            raise ValueError(f"name already exists: {name}")
        d = Dataset(data, **options)
        self._children[name] = d
        return d

    def keys(self):
        return self._children.keys()

    def __iter__(self):
        return iter(self._children)

    def __contains__(self, name):
        return name in self._children

    def __getitem__(self, name):
        return self._children[name]


class File(Group):
    def __init__(self, path, mode="r"):
        super().__init__()
        self._path, self._mode = Path(path), mode
        if mode in ("r", "r+"):
            try:
                root = pickle.loads(self._path.read_bytes())
            except (pickle.UnpicklingError, EOFError, ValueError) as error:
                raise OSError(f"unable to open file (not an archive): {error}") from error
            self.attrs, self._children = root.attrs, root._children
        elif mode != "w":
            raise ValueError(f"unsupported mode {mode}")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        if self._mode in ("w", "r+"):
            root = Group()
            root.attrs, root._children = self.attrs, self._children
            self._path.write_bytes(pickle.dumps(root))
        return False
