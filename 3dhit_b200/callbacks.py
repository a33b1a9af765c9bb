"""Callbacks for `evolve` (reference: src/hit3d/callbacks.py).

Same scheduling rules as the reference (callbacks.py:43-104): wrappers carry
``every`` or ``every_time``, fire at step 0, and callback functions are pure
observers of a `State`.  HDF5 persistence (``FieldWriter``, ``save_series``)
needs h5py, which is optional: without it those two raise ImportError.
"""

from __future__ import annotations

import math
import os
from typing import NamedTuple

import numpy as np
import torch

__all__ = ["State", "Callback", "Diagnostic", "FieldWriter", "save_series"]


class State(NamedTuple):
    """Read-only snapshot handed to callback functions (callbacks.py:33-40)."""

    u_hat: object
    t: float
    step: int
    params: object
    grid: object


def _host(v):
    if isinstance(v, dict):
        return {k: _host(x) for k, x in v.items()}
    if isinstance(v, torch.Tensor):
        v = v.detach().cpu()
        return v.item() if v.ndim == 0 else v.numpy()
    return v


class Callback:
    """callbacks.py:43-66."""

    def __init__(self, f, *, every=1, every_time=None):
        self.f = f
        self.every = every
        self.every_time = every_time

    def is_due(self, step, t, dt):
        if self.every_time is None:
            return step % self.every == 0
        return step == 0 or (math.floor(t / self.every_time) > math.floor((t - dt) / self.every_time))

    def fire(self, state):
        self.f(state)

    def finalize(self):
        pass


class Diagnostic:
    """Time-series recorder (callbacks.py:69-104); values are pulled to the
    host on every fire."""

    def __init__(self, f, *, every=1, path=None, name=None):
        if path is not None and name is None:
            raise ValueError("Diagnostic(..., path=...) also needs `name` "
                             "(the series/<name> group to persist it under)")
        self.f = f
        self.every = every
        self.path = path
        self.name = name
        self.times = []
        self.values = []

    def is_due(self, step, t, dt):
        return step % self.every == 0

    def fire(self, state):
        self.times.append(float(state.t))
        self.values.append(_host(self.f(state)))

    def finalize(self):
        if self.path is not None:
            save_series(self.path, self.name, self)


def _h5py():
    try:
        import h5py
    except ImportError as e:  # optional dependency, as in the reference's IO layer
        raise ImportError("FieldWriter/save_series need h5py") from e
    return h5py


class FieldWriter:
    """Full-field snapshot writer (callbacks.py:108-185), same HDF5 layout
    (``grid/*``, ``step_%08d/{t,u_hat}``)."""

    def __init__(self, path, *, every=1, fields=("u_hat",), overwrite=True, every_time=None,
                 warmup_time=None):
        _h5py()
        if every_time is not None and warmup_time is None:
            warmup_time = 0.0
        d = os.path.dirname(path)
        if d:
            os.makedirs(d, exist_ok=True)
        if overwrite and os.path.exists(path):
            os.remove(path)
        self.path = path
        self.every = every
        self.fields = tuple(fields)
        self.every_time = every_time
        self.warmup_time = warmup_time

    def is_due(self, step, t, dt):
        if self.every_time is None:
            return step % self.every == 0
        if t < self.warmup_time:
            return False
        tol = (dt / self.every_time) / 4

        def index(x):
            r = round(x)
            return r if abs(x - r) < tol else x

        n_now = math.floor(index((t - self.warmup_time) / self.every_time))
        n_prev = math.floor(index((t - dt - self.warmup_time) / self.every_time))
        return n_now > n_prev

    def fire(self, state):
        h5py = _h5py()
        with h5py.File(self.path, "a") as f:
            if "grid/Nx" not in f:
                g = state.grid
                for name, val in (("Nx", g.Nx), ("Ny", g.Ny), ("Nz", g.Nz),
                                  ("Lx", g.Lx), ("Ly", g.Ly), ("Lz", g.Lz)):
                    f[f"grid/{name}"] = val
                nu = getattr(state.params, "nu", None)
                if nu is not None:
                    f["grid/nu"] = float(nu)
            grp = f"step_{state.step:08d}"
            f[f"{grp}/t"] = float(state.t)
            for fld in self.fields:
                f[f"{grp}/{fld}"] = np.asarray(_host(getattr(state, fld)))

    def finalize(self):
        pass


def save_series(path, name, diagnostic):
    """Columnar series under ``series/<name>/`` (callbacks.py:188-217)."""
    h5py = _h5py()
    with h5py.File(path, "a") as f:
        key = f"series/{name}"
        if key in f:
            raise ValueError(f"{key} already exists in {path} (saving the same series twice? "
                             "reruns should start from a fresh file)")
        f[f"{key}/t"] = np.asarray(diagnostic.times)
        values = diagnostic.values
        if values and isinstance(values[0], dict):
            for fld in values[0]:
                f[f"{key}/{fld}"] = np.asarray([v[fld] for v in values])
        else:
            f[f"{key}/values"] = np.asarray(values)
    return path
