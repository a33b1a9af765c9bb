"""Callbacks for `evolve` (reference interface: src/hit3d/callbacks.py:33-217).

The interface is the reference's: a callback object answers
``is_due(step, t, dt)``, is handed a read-only `State` by ``fire`` and is told
``finalize()`` when the run ends; `Callback`, `Diagnostic` and `FieldWriter`
take the reference's arguments and keep its schedules, and files follow the
HDF5 layout of `schema`.  What differs is how the work meets the GPU:

* `Diagnostic` keeps small device results (a budget, a spectrum) on the
  device and brings everything recorded so far to the host in one batched
  transfer when ``values`` is read or the run ends, instead of one
  synchronising read per firing, so rollout segments follow each other
  without host round trips.
* `FieldWriter` copies a snapshot into reused pinned host buffers on a side
  stream and writes it to HDF5 at its next firing or at the end of the run,
  so the file write overlaps the next rollout segment.

HDF5 needs h5py, which is optional: without it `FieldWriter` and
`save_series` raise ImportError.
"""

from __future__ import annotations

import math
import os
from typing import NamedTuple

import numpy as np
import torch

from .schema import grid_key, series_field, series_key, step_key

__all__ = ["State", "Callback", "Diagnostic", "FieldWriter", "save_series"]


class State(NamedTuple):
    """What a callback function sees: the state at one step, read-only."""

    u_hat: object
    t: float
    step: int
    params: object
    grid: object


def _cadence_index(t, period, offset=0.0, slack=0.0):
    """Index of the last time offset + k*period at or before t; `slack` (in
    periods) lets a time that falls just short of a multiple through
    rounding count as reaching it."""
    return math.floor((t - offset) / period + slack)


def _crossed(t, dt, period, offset=0.0, slack=0.0):
    """Whether the step (t - dt, t] reaches a new multiple of `period`."""
    return _cadence_index(t, period, offset, slack) > _cadence_index(t - dt, period, offset, slack)


class Callback:
    """Calls ``f(state)`` on its schedule and drops the result: every
    `every` steps, or, when `every_time` is set, at step 0 and on every step
    that crosses a multiple of `every_time` in simulation time."""

    def __init__(self, f, *, every=1, every_time=None):
        self.f = f
        self.every = every
        self.every_time = every_time

    def is_due(self, step, t, dt):
        if self.every_time is not None:
            return step == 0 or _crossed(t, dt, self.every_time)
        return step % self.every == 0

    def fire(self, state):
        self.f(state)

    def finalize(self):
        pass


def _to_host_batched(leaves):
    """Host copies of CUDA tensors with one transfer per (device, dtype): the
    leaves are flattened into one device buffer each, copied into pinned
    memory and split again."""
    out = [None] * len(leaves)
    groups = {}
    for i, t in enumerate(leaves):
        groups.setdefault((t.device, t.dtype), []).append(i)
    events = []
    for (dev, _), idx in groups.items():
        flat = torch.cat([leaves[i].reshape(-1) for i in idx])
        host = flat.to("cpu", non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(torch.cuda.current_stream(dev))
        events.append((ev, host, idx))
    for ev, host, idx in events:
        ev.synchronize()
        off = 0
        for i in idx:
            n = leaves[i].numel()
            out[i] = host[off:off + n].reshape(leaves[i].shape)
            off += n
    return out


class _Leaf:
    __slots__ = ("i",)

    def __init__(self, i):
        self.i = i


def _host_value(v):
    """A host copy of one value (scalars for 0-d tensors)."""
    if isinstance(v, torch.Tensor):
        v = v.detach().cpu()
        return v.item() if v.ndim == 0 else v.numpy()
    return v


class Diagnostic:
    """Time-series recorder: ``f(state)`` (a scalar, an array or a dict of
    them) and the time at every `every`-th step, step 0 included.  ``times``
    and ``values`` hold the series on the host; with `path` and `name` it is
    saved under ``series/<name>`` of that file when the run ends.

    Device results of up to `DEFER_LIMIT` bytes per firing stay on the device
    until ``values`` is read or the run finishes, then come over in one
    transfer; larger ones are copied at once (they would pin device memory)."""

    DEFER_LIMIT = 1 << 20

    def __init__(self, f, *, every=1, path=None, name=None):
        if path is not None and name is None:
            raise ValueError("a Diagnostic saved to a file needs the series name too: "
                             "Diagnostic(f, path=..., name=...)")
        self.f = f
        self.every = every
        self.path = path
        self.name = name
        self.times = []
        self._values = []
        self._pending = []  # device results not yet on the host, in firing order

    def is_due(self, step, t, dt):
        return step % self.every == 0

    def fire(self, state):
        v = self.f(state)
        self.times.append(float(state.t))
        if self._pending or _device_bytes(v) > 0:
            self._pending.append(v)
            if _device_bytes(v) > self.DEFER_LIMIT:
                self._fetch()
        else:
            self._values.append(_host_tree(v))

    @property
    def values(self):
        self._fetch()
        return self._values

    def _fetch(self):
        if not self._pending:
            return
        leaves = []

        def strip(v):
            if isinstance(v, dict):
                return {k: strip(x) for k, x in v.items()}
            if isinstance(v, (list, tuple)):
                return type(v)(strip(x) for x in v)
            if isinstance(v, torch.Tensor) and v.is_cuda:
                leaves.append(v.detach())
                return _Leaf(len(leaves) - 1)
            return _host_value(v)

        shapes = [strip(v) for v in self._pending]
        host = _to_host_batched(leaves)

        def fill(s):
            if isinstance(s, dict):
                return {k: fill(x) for k, x in s.items()}
            if isinstance(s, (list, tuple)):
                return type(s)(fill(x) for x in s)
            if isinstance(s, _Leaf):
                t = host[s.i]
                return t.item() if t.ndim == 0 else t.numpy()
            return s

        self._values.extend(fill(s) for s in shapes)
        self._pending = []

    def finalize(self):
        self._fetch()
        if self.path is not None:
            save_series(self.path, self.name, self)


def _device_bytes(v):
    if isinstance(v, dict):
        return sum(_device_bytes(x) for x in v.values())
    if isinstance(v, (list, tuple)):
        return sum(_device_bytes(x) for x in v)
    if isinstance(v, torch.Tensor) and v.is_cuda:
        return max(v.numel() * v.element_size(), 1)
    return 0


def _host_tree(v):
    if isinstance(v, dict):
        return {k: _host_tree(x) for k, x in v.items()}
    return _host_value(v)


def _h5py():
    try:
        import h5py
    except ImportError as e:  # optional: only the HDF5 writers need it
        raise ImportError("FieldWriter and save_series write HDF5 and need h5py") from e
    return h5py


class FieldWriter:
    """Snapshots of state fields (``u_hat`` by default) in an HDF5 file, one
    ``step_<n>`` group each with the time, plus the grid (and ``nu``) in
    ``grid/`` on the first write.  Scheduled every `every` steps, or, with
    `every_time`, at ``warmup_time`` (default 0) and every `every_time` of
    simulation time after it, none before.  ``overwrite=True`` (default)
    deletes an existing file when the writer is made.

    A due snapshot is copied device -> pinned host memory on a side stream;
    its HDF5 write happens at the next firing or at ``finalize``, so it
    overlaps the rollout segment in between."""

    def __init__(self, path, *, every=1, fields=("u_hat",), overwrite=True, every_time=None, warmup_time=None):
        _h5py()
        self.path = path
        self.every = every
        self.fields = tuple(fields)
        self.every_time = every_time
        # a time cadence starts at warmup_time, by default at t = 0
        self.warmup_time = 0.0 if every_time is not None and warmup_time is None else warmup_time
        parent = os.path.dirname(path)
        if parent:
            os.makedirs(parent, exist_ok=True)
        if overwrite and os.path.exists(path):
            os.remove(path)
        self._pinned = {}   # field -> reused pinned host buffer
        self._staged = None  # (state, {field: host array or pinned tensor}, event)
        self._side = None

    def is_due(self, step, t, dt):
        if self.every_time is None:
            return step % self.every == 0
        if t < self.warmup_time:
            return False
        # t = t0 + n dt is rounded differently from the (t - dt) formed here, so
        # times within a quarter step of a cadence point count as reaching it
        return _crossed(t, dt, self.every_time, self.warmup_time, slack=dt / (4 * self.every_time))

    def _buffer(self, fld, v):
        b = self._pinned.get(fld)
        if b is None or b.shape != v.shape or b.dtype != v.dtype:
            b = torch.empty(v.shape, dtype=v.dtype, pin_memory=True)
            self._pinned[fld] = b
        return b

    def fire(self, state):
        self._write_staged()
        copies, event = {}, None
        for fld in self.fields:
            v = getattr(state, fld)
            if isinstance(v, torch.Tensor) and v.is_cuda:
                if self._side is None or self._side.device != v.device:
                    self._side = torch.cuda.Stream(device=v.device)
                buf = self._buffer(fld, v)
                self._side.wait_stream(torch.cuda.current_stream(v.device))
                with torch.cuda.stream(self._side):
                    buf.copy_(v, non_blocking=True)
                v.record_stream(self._side)  # the producer's memory stays allocated until the copy ends
                event = torch.cuda.Event()
                event.record(self._side)
                copies[fld] = buf
            else:
                copies[fld] = np.array(_host_value(v))
        self._staged = (state, copies, event)

    def _write_staged(self):
        if self._staged is None:
            return
        state, copies, event = self._staged
        self._staged = None
        if event is not None:
            event.synchronize()
        h5py = _h5py()
        with h5py.File(self.path, "a") as f:
            if "grid" not in f:
                g = state.grid
                for key in ("Nx", "Ny", "Nz", "Lx", "Ly", "Lz"):
                    f[grid_key(key)] = getattr(g, key)
                nu = getattr(state.params, "nu", None)
                if nu is not None:
                    f[grid_key("nu")] = float(nu)
            grp = step_key(state.step)
            f[grp + "/t"] = float(state.t)
            for fld, host in copies.items():
                f[grp + "/" + fld] = host.numpy() if isinstance(host, torch.Tensor) else host

    def finalize(self):
        self._write_staged()


def save_series(path, name, diagnostic):
    """Write a `Diagnostic`'s series into the HDF5 file at `path` under
    ``series/<name>/``: the times as ``t`` and the values as one ``values``
    column, or one column per key of dict values.  The file is appended to
    (typically the run's snapshot file); an existing ``series/<name>`` is an
    error."""
    h5py = _h5py()
    values = diagnostic.values
    if values and isinstance(values[0], dict):
        cols = {k: np.asarray([v[k] for v in values]) for k in values[0]}
    else:
        cols = {"values": np.asarray(values)}
    with h5py.File(path, "a") as f:
        if series_key(name) in f:
            raise ValueError(f"{path} already holds {series_key(name)}; each series is saved once per file "
                             "(start a rerun from a fresh file)")
        f[series_field(name, "t")] = np.asarray(diagnostic.times)
        for k, col in cols.items():
            f[series_field(name, k)] = col
    return path
