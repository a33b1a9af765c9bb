"""Discrete adjoint of the RHS, the RK4 step and the rollout.

The reference differentiates ``rhs``, ``rk4_step`` and ``rollout``
(src/hit3d/navierstokes.py:62-97, src/hit3d/integrators.py:32-53) with
``jax.vjp``/``jax.grad`` through XLA.  Here the transposes are written out
and run on the GPU (``hit_rhs_vjp``, ``hit_rk4_step_vjp``, ``hit_rollout_vjp``
in include/hit3d.h):

* ``rhs_vjp``, ``rk4_step_vjp``, ``rollout_vjp`` return the cotangent of the
  state and a dict of parameter cotangents ``{"nu", "A", "eps"}`` (``A`` of
  ``LinearForcing``, ``eps`` of ``BandForcing``);
* ``rollout_autograd`` is a ``torch.autograd.Function`` around ``rollout``
  whose backward is ``rollout_vjp``: gradients reach the initial state and the
  parameters given as 0-dim tensors.

Cotangents are dL/dRe + i dL/dIm of the stored half-spectrum entries, which
is PyTorch's convention for complex tensors (``jax.vjp`` returns the complex
conjugate).  The rollout keeps a state every ``checkpoint_every`` steps and
recomputes each segment, so memory is (nsteps / K + K) states.
"""

from __future__ import annotations

import torch

from . import _native as nat
from .forcing import BandForcing, LinearForcing, native_params
from .grid import _check_state
from .integrators import rollout
from .navierstokes import NSParams, NSRHS

__all__ = ["rhs_vjp", "rk4_step_vjp", "rollout_vjp", "rollout_autograd", "PARAM_NAMES"]

PARAM_NAMES = ("nu", "A", "eps")


def _setup(rhs, params, u_hat, ct):
    if not isinstance(rhs, NSRHS):
        raise ValueError("the adjoint needs the package's own RHS (make_ns_rhs)")
    p = native_params(params.nu, params.forcing)
    if p is None:
        raise ValueError("the adjoint supports the built-in forcings only")
    g = rhs.grid
    u_hat = _check_state(u_hat, g)
    ct = _check_state(ct, g)
    return g, p, u_hat, ct


def _params_dict(pct):
    vals = pct.tolist()
    return dict(zip(PARAM_NAMES, vals))


def rhs_vjp(rhs, u_hat, params, ct, t=0.0):
    """(d rhs / d u_hat)^T ct and the parameter cotangents."""
    g, p, u_hat, ct = _setup(rhs, params, u_hat, ct)
    out = torch.empty_like(u_hat)
    pct = torch.zeros(3, dtype=torch.float64, device=u_hat.device)
    nat.call("hit_rhs_vjp", g.plan.handle, nat.ptr(u_hat), p, float(t), nat.ptr(ct), nat.ptr(out), nat.ptr(pct),
             nat.stream_ptr(g.device))
    return out, _params_dict(pct)


def rk4_step_vjp(rhs, u_hat, params, dt, ct, t=0.0):
    """(d rk4_step / d u_hat)^T ct (stage inputs recomputed) and the parameter
    cotangents."""
    g, p, u_hat, ct = _setup(rhs, params, u_hat, ct)
    out = torch.empty_like(u_hat)
    pct = torch.zeros(3, dtype=torch.float64, device=u_hat.device)
    nat.call("hit_rk4_step_vjp", g.plan.handle, nat.ptr(u_hat), p, float(dt), float(t), nat.ptr(ct), nat.ptr(out),
             nat.ptr(pct), nat.stream_ptr(g.device))
    return out, _params_dict(pct)


def rollout_vjp(rhs, u0, params, dt, nsteps, ct, t0=0.0, checkpoint_every=20):
    """(d rollout / d u0)^T ct with checkpoints every ``checkpoint_every``
    steps, and the parameter cotangents summed over the steps."""
    g, p, u0, ct = _setup(rhs, params, u0, ct)
    out = torch.empty_like(u0)
    pct = torch.zeros(3, dtype=torch.float64, device=u0.device)
    nat.call("hit_rollout_vjp", g.plan.handle, nat.ptr(u0), p, float(dt), int(nsteps), float(t0),
             int(checkpoint_every), nat.ptr(ct), nat.ptr(out), nat.ptr(pct), nat.stream_ptr(g.device))
    return out, _params_dict(pct)


def _with_values(params, nu, A, eps):
    f = params.forcing
    if isinstance(f, LinearForcing):
        f = LinearForcing(A=float(A))
    elif isinstance(f, BandForcing):
        f = BandForcing(eps=float(eps), kmin=f.kmin, kmax=f.kmax)
    return NSParams(nu=float(nu), forcing=f)


class _Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u0, nu, A, eps, rhs, params, dt, nsteps, checkpoint_every):
        prm = _with_values(params, nu, A, eps)
        ctx.rhs, ctx.params, ctx.dt, ctx.nsteps, ctx.K = rhs, prm, dt, nsteps, checkpoint_every
        ctx.save_for_backward(u0)
        return rollout(rhs, u0.detach(), prm, dt, nsteps, assume_dealiased=False)

    @staticmethod
    def backward(ctx, ct):
        (u0,) = ctx.saved_tensors
        ub, pb = rollout_vjp(ctx.rhs, u0.detach(), ctx.params, ctx.dt, ctx.nsteps, ct.contiguous(),
                             checkpoint_every=ctx.K)
        dev = u0.device
        grads = [torch.tensor(pb[k], dtype=torch.float64, device=dev) for k in PARAM_NAMES]
        return (ub, *grads, None, None, None, None, None)


def rollout_autograd(rhs, u0, params, dt, nsteps, checkpoint_every=20):
    """``rollout`` that torch autograd differentiates through the hand-written
    adjoint.  ``params.nu`` and the forcing's ``A`` / ``eps`` may be 0-dim
    tensors with ``requires_grad``; their gradients are float64."""
    f = params.forcing

    def scalar(x):
        return x if isinstance(x, torch.Tensor) else torch.tensor(float(x), dtype=torch.float64)

    nu = scalar(params.nu)
    A = scalar(getattr(f, "A", 0.0))
    eps = scalar(getattr(f, "eps", 0.0))
    return _Rollout.apply(u0, nu, A, eps, rhs, params, float(dt), int(nsteps), int(checkpoint_every))
