"""Recording stand-in for h5py -- TEST INFRASTRUCTURE ONLY.

h5py is installed neither here nor on the GPU machines, so a writer's HDF5
output is checked through this stand-in: ``File`` behaves like h5py.File for
what a tree-brick writer uses (create_group, [] on groups, attrs, and
create_dataset with data or a shape plus slice assignment) and records every
call in order.  ``record_of(f)`` turns the log into a JSON-able list plus the
arrays it holds, so a record of the reference's writer can be stored as a
fixture and compared with a record of this library's writer.
"""
from __future__ import annotations

import numpy as np


def _value(v):
    if isinstance(v, np.ndarray):
        return {"t": "ndarray", "dtype": str(v.dtype), "v": v.tolist()}
    if isinstance(v, (bool, np.bool_)):
        return {"t": type(v).__name__, "v": bool(v)}
    if isinstance(v, (int, np.integer)):
        return {"t": type(v).__name__, "v": int(v)}
    if isinstance(v, (float, np.floating)):
        return {"t": type(v).__name__, "v": repr(float(v))}
    if isinstance(v, str):
        return {"t": "str", "v": v}
    raise TypeError(f"attribute value of type {type(v)}")


class _Attrs:
    def __init__(self, log, path):
        self._log, self._path = log, path

    def __setitem__(self, name, value):
        self._log.append({"op": "attr", "path": self._path, "name": name, "value": _value(value)})


class _Dataset:
    def __init__(self, log, path):
        self._log, self._path = log, path
        self.attrs = _Attrs(log, path)

    def __setitem__(self, key, value):
        self._log.append({"op": "write", "path": self._path, "key": repr(key), "data": np.array(value, copy=True)})


class _Group:
    def __init__(self, log, path):
        self._log, self._path = log, path
        self.attrs = _Attrs(log, path)
        self._children = {}

    def create_group(self, name):
        p = f"{self._path}/{name}"
        self._log.append({"op": "group", "path": p})
        g = _Group(self._log, p)
        self._children[name] = g
        return g

    def __getitem__(self, name):
        return self._children[name]

    def create_dataset(self, name, shape=None, dtype=None, data=None, **kw):
        p = f"{self._path}/{name}"
        self._log.append({"op": "dataset", "path": p, "shape": None if shape is None else list(shape),
                          "dtype": None if dtype is None else str(np.dtype(dtype)),
                          "data": None if data is None else np.array(data, copy=True),
                          "kw": {k: (list(v) if isinstance(v, tuple) else v) for k, v in sorted(kw.items())}})
        d = _Dataset(self._log, p)
        self._children[name] = d
        return d


class File(_Group):
    """h5py.File stand-in; the file on disk is created empty (writers chmod it)."""

    opened: list = []

    def __init__(self, name, mode="r"):
        super().__init__([], "")
        self.filename, self.mode = name, mode
        if "w" in mode:
            open(name, "wb").close()
        File.opened.append(self)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def record_of(f):
    """(JSON-able log, {key: array}) of a stand-in File's calls."""
    log, arrays = [], {}
    for k, e in enumerate(f._log):
        e = dict(e)
        if isinstance(e.get("data"), np.ndarray):
            key = f"d{k}"
            arrays[key] = e["data"]
            e["data"] = key
        log.append(e)
    return log, arrays
