"""A minimal in-memory stand-in for ``h5py`` (absent here): enough of
``h5py.File`` for the HDF5 writers and the tests that read their files back.

Datasets live in a module-level dict per path; the path also exists on disk
(an empty marker file), so ``os.path.exists``/``os.remove`` see it, and a
file deleted on disk starts empty when reopened.  Keys are '/'-separated;
``key in f`` is true for datasets and for the groups above them; ``f[key]``
returns a `Dataset` (``[()]`` gives the value) or a `Group`; iterating a file
or group yields its direct children."""

from __future__ import annotations

import os

import numpy as np

_FILES: dict[str, dict[str, np.ndarray]] = {}


class Dataset:
    def __init__(self, value):
        self._v = value

    def __getitem__(self, idx):
        return self._v[idx] if idx != () else self._v[()]


class Group:
    def __init__(self, store, prefix):
        self._s, self._p = store, prefix

    def _children(self):
        pre = self._p + "/" if self._p else ""
        return sorted({k[len(pre):].split("/")[0] for k in self._s if k.startswith(pre)})

    def __iter__(self):
        return iter(self._children())

    def keys(self):
        return self._children()

    def __contains__(self, key):
        full = f"{self._p}/{key}" if self._p else key
        return full in self._s or any(k.startswith(full + "/") for k in self._s)

    def __getitem__(self, key):
        full = f"{self._p}/{key}" if self._p else key
        if full in self._s:
            return Dataset(self._s[full])
        if any(k.startswith(full + "/") for k in self._s):
            return Group(self._s, full)
        raise KeyError(key)

    def __setitem__(self, key, value):
        full = f"{self._p}/{key}" if self._p else key
        if full in self._s or any(k.startswith(full + "/") for k in self._s):
            raise ValueError(f"name already exists: {full}")
        self._s[full] = np.asarray(value)


class File(Group):
    def __init__(self, path, mode="r"):
        path = os.path.abspath(path)
        if not os.path.exists(path):
            if mode == "r":
                raise FileNotFoundError(path)
            _FILES[path] = {}
            open(path, "w").close()
        super().__init__(_FILES.setdefault(path, {}), "")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def close(self):
        pass
