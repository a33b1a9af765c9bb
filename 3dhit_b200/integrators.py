"""Time integration (reference: src/hit3d/integrators.py).

``rk4_step`` and ``rollout`` with the package's own RHS and a built-in
forcing run entirely in the fused kernels: the rollout is one launch of a CUDA
graph whose while node loops over the ``nsteps`` steps on the device, on the
current stream with no host synchronisation (the replacement for the jitted
``lax.scan``).  Any other
``rhs`` callable is integrated by composing its calls with the reference's
stage algebra.  ``evolve`` is the host loop over rollout segments with
callbacks (reference interface: integrators.py:56-109).
"""

from __future__ import annotations

import time

import torch

from . import _native as nat
from .callbacks import State
from .forcing import native_params
from .grid import _check_state
from .navierstokes import NSRHS, resolve_flags

__all__ = ["rk4_step", "ifrk4_step", "rollout", "evolve", "SCHEMES"]

SCHEMES = ("rk4", "ifrk4")


def _as_tensor(rhs, u_hat):
    if isinstance(u_hat, torch.Tensor):
        return u_hat
    g = getattr(rhs, "grid", None)
    if g is not None:
        return _check_state(u_hat, g)
    return torch.as_tensor(u_hat, device="cuda")


def _fused(rhs, params):
    return isinstance(rhs, NSRHS) and native_params(params.nu, params.forcing) is not None


def _flags(u_hat, g, assume_dealiased, scheme):
    if scheme not in SCHEMES:
        raise ValueError(f"unknown scheme {scheme!r}; expected one of {SCHEMES}")
    f = resolve_flags(u_hat, g, assume_dealiased)
    return f | nat.HIT_FLAG_INTEGRATING_FACTOR if scheme == "ifrk4" else f


def rk4_step(rhs, u_hat, params, dt, t, *, assume_dealiased=None, scheme="rk4", f_ext=None, out=None):
    """One classic RK4 step (integrators.py:32-38); ``scheme="ifrk4"`` takes
    the integrating-factor step of `ifrk4_step` instead.  ``f_ext``: an
    external force held over the step (see `NSRHS.__call__`).  ``out``: a
    state-shaped tensor (not ``u_hat``) that receives the new state."""
    if out is not None and out.data_ptr() == u_hat.data_ptr():
        raise ValueError("out must not alias u_hat")
    if _fused(rhs, params):
        g = rhs.grid
        u_hat = _check_state(u_hat, g)
        p = native_params(params.nu, params.forcing, _flags(u_hat, g, assume_dealiased, scheme))
        if out is None:
            out = torch.empty_like(u_hat)
        elif out.shape != u_hat.shape or out.dtype != u_hat.dtype or not out.is_contiguous():
            raise ValueError("out must be a contiguous tensor of the state's shape and dtype")
        if f_ext is not None:
            f_ext = _check_state(f_ext, g)
            nat.call("hit_rollout_forced", g.plan.handle, nat.ptr(u_hat), p, nat.ptr(f_ext), float(dt), 1,
                     float(t), nat.ptr(out), nat.stream_ptr(g.device))
        else:
            nat.call("hit_rk4_step", g.plan.handle, nat.ptr(u_hat), p, float(dt), float(t), nat.ptr(out),
                     nat.stream_ptr(g.device))
        return out
    if f_ext is not None:
        base = rhs
        if not isinstance(base, NSRHS):
            raise ValueError("f_ext needs the package's RHS (make_ns_rhs)")

        def rhs(u, p, tt):
            return base(u, p, tt, f_ext=f_ext)
        rhs.grid = base.grid
    if out is not None:
        return out.copy_(rk4_step(rhs, u_hat, params, dt, t, assume_dealiased=assume_dealiased, scheme=scheme,
                                  f_ext=f_ext))
    if scheme == "ifrk4":
        return _ifrk4_composed(rhs, u_hat, params, dt, t)
    if scheme != "rk4":
        raise ValueError(f"unknown scheme {scheme!r}; expected one of {SCHEMES}")
    u_hat = _as_tensor(rhs, u_hat)
    k1 = rhs(u_hat, params, t)
    k2 = rhs(u_hat + 0.5 * dt * k1, params, t + 0.5 * dt)
    k3 = rhs(u_hat + 0.5 * dt * k2, params, t + 0.5 * dt)
    k4 = rhs(u_hat + dt * k3, params, t + dt)
    return u_hat + (dt / 6.0) * (k1 + 2 * k2 + 2 * k3 + k4)


def ifrk4_step(rhs, u_hat, params, dt, t, *, assume_dealiased=None):
    """One integrating-factor (Lawson) RK4 step on the viscous operator
    ``linear_operator(grid, params) = -nu k^2`` (navierstokes.py:100-103), the
    scheme the reference lists as to do (integrators.py:15-16).  With
    E = exp(-nu k^2 dt/2) and N the RHS without its viscous term:

        k1 = N(u),  k2 = N(E (u + dt/2 k1)),  k3 = N(E u + dt/2 k2),
        k4 = N(E^2 u + dt E k3),
        u' = E^2 u + dt/6 ((E (E k1 + 2 k2) + 2 E k3) + k4).

    The viscous decay is exact, so the step is not limited by nu k^2 dt; for
    a Beltrami field (u x w = 0) it reproduces exp(-nu k^2 t) u exactly.  With
    the package's RHS and a built-in forcing it runs in the fused kernels at
    the cost of an RK4 step."""
    return rk4_step(rhs, u_hat, params, dt, t, assume_dealiased=assume_dealiased, scheme="ifrk4")


def _ifrk4_composed(rhs, u_hat, params, dt, t):
    """`ifrk4_step` for an RHS the fused kernels cannot run (a custom forcing
    or another callable with a ``grid``): N(v) = rhs(v) - L v."""
    from .navierstokes import linear_operator
    g = getattr(rhs, "grid", None)
    if g is None:
        raise ValueError("ifrk4 needs rhs.grid for the linear operator")
    u_hat = _as_tensor(rhs, u_hat)
    L = linear_operator(g, params).to(u_hat.device)
    E = torch.exp((0.5 * dt) * L)

    def N(v, tt):
        return rhs(v, params, tt) - L * v

    k1 = N(u_hat, t)
    k2 = N(E * (u_hat + 0.5 * dt * k1), t + 0.5 * dt)
    k3 = N(E * u_hat + 0.5 * dt * k2, t + 0.5 * dt)
    ek3 = E * k3
    k4 = N((E * E) * u_hat + dt * ek3, t + dt)
    return (E * E) * u_hat + (dt / 6.0) * ((E * (E * k1 + 2 * k2) + 2 * ek3) + k4)


def rollout(rhs, u_hat, params, dt, nsteps, t0=0.0, *, assume_dealiased=None, scheme="rk4", f_ext=None):
    """Advance `nsteps` RK4 steps (integrators.py:41-53), or integrating-factor
    RK4 steps (`ifrk4_step`) with ``scheme="ifrk4"``; ``f_ext``: an external
    force held over the whole rollout."""
    nsteps = int(nsteps)
    if _fused(rhs, params):
        g = rhs.grid
        u_hat = _check_state(u_hat, g)
        p = native_params(params.nu, params.forcing, _flags(u_hat, g, assume_dealiased, scheme))
        out = torch.empty_like(u_hat)
        if f_ext is not None:
            f_ext = _check_state(f_ext, g)
            nat.call("hit_rollout_forced", g.plan.handle, nat.ptr(u_hat), p, nat.ptr(f_ext), float(dt), nsteps,
                     float(t0), nat.ptr(out), nat.stream_ptr(g.device))
        else:
            nat.call("hit_rollout", g.plan.handle, nat.ptr(u_hat), p, float(dt), nsteps, float(t0),
                     nat.ptr(out), nat.stream_ptr(g.device))
        return out
    for i in range(nsteps):
        u_hat = rk4_step(rhs, u_hat, params, dt, t0 + i * dt, scheme=scheme, f_ext=f_ext)
    return u_hat


def _progress_interval(progress, nsteps):
    """Steps between progress lines: 0 = silent; True = about 20 lines."""
    if progress is True:
        return max(nsteps // 20, 1)
    if progress is False or progress is None:
        return 0
    return max(int(progress), 1)


class _ProgressLine:
    """One line per report: step, percentage, simulation time, wall time, an
    estimate of the time left and the step rate."""

    def __init__(self, nsteps):
        self.nsteps = nsteps
        self.start = time.perf_counter()

    @staticmethod
    def _clock(sec):
        m, s = divmod(sec, 60.0)
        return f"{s:.1f}s" if m == 0 else f"{int(m)}m{int(round(s)):02d}s"

    def report(self, n, t):
        wall = time.perf_counter() - self.start
        left = wall * (self.nsteps - n) / n
        pct = int(round(100.0 * n / self.nsteps))
        print(f"step {n}/{self.nsteps} ({pct:3d}%)  t = {t:.6g}  wall {self._clock(wall)}  "
              f"eta {self._clock(left)}  [{n / max(wall, 1e-9):.1f} steps/s]", flush=True)


def _firing_plan(callbacks, nsteps, t0, dt):
    """{step: callbacks due at that step}, asking each callback once per step
    (the step's time is t0 + n dt, as the rollout segments see it)."""
    plan = {}
    for n in range(nsteps + 1):
        t = t0 + n * dt
        due = [cb for cb in callbacks if cb.is_due(n, t, dt)]
        if due:
            plan[n] = due
    return plan


def evolve(rhs, u_hat, params, grid, dt, nsteps, *, t0=0.0, callbacks=(), progress=False, scheme="rk4"):
    """Advance `nsteps` steps while firing callbacks (reference interface:
    src/hit3d/integrators.py:56-109; ``scheme`` as in `rollout`).

    The firing plan is made up front (each callback asked once per step);
    the run is then a chain of `rollout` segments, each ending on a step
    where a callback fires or a progress line is due, and callbacks see a
    `State` of that step.  No host synchronisation is added between segments:
    `Diagnostic` defers its device reads and `FieldWriter` stages snapshots
    through pinned memory, so the GPU runs the segments back to back.  At the
    end every callback is finalised and the transform kernels' wait flag is
    checked (raises `DeviceWaitError` if a bounded wait gave up)."""
    nsteps = int(nsteps)
    every = _progress_interval(progress, nsteps)
    plan = _firing_plan(callbacks, nsteps, t0, dt)
    stops = set(plan) | ({nsteps} if nsteps > 0 else set())
    if every:
        stops |= set(range(every, nsteps + 1, every))
    stops.discard(0)
    line = _ProgressLine(nsteps) if every else None

    def fire(n, u):
        for cb in plan.get(n, ()):
            cb.fire(State(u_hat=u, t=t0 + n * dt, step=n, params=params, grid=grid))

    fire(0, u_hat)
    done = 0
    dealiased = None  # decided once (one device check) for the fused path
    for n in sorted(stops):
        if dealiased is None and _fused(rhs, params):
            dealiased = bool(resolve_flags(_check_state(u_hat, grid), grid, None))
        u_hat = rollout(rhs, u_hat, params, dt, n - done, t0 + done * dt, assume_dealiased=dealiased, scheme=scheme)
        fire(n, u_hat)
        if line is not None and (n % every == 0 or n == nsteps):
            line.report(n, t0 + n * dt)
        done = n
    for cb in callbacks:
        cb.finalize()
    if isinstance(u_hat, torch.Tensor) and u_hat.is_cuda:
        with torch.cuda.device(u_hat.device):
            nat.check_device("evolve")
    return u_hat
