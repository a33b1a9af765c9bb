"""Navier-Stokes RHS in rotational form (reference: src/hit3d/navierstokes.py).

    du/dt = P(k) [ (u x w)^ + f ] - nu k^2 u

``make_ns_rhs(grid)`` returns ``rhs(u_hat, params, t)``; with a built-in
forcing one call is one pass chain of the fused sm_100a kernels
(``hit_rhs``).  A custom forcing object is added through the identity
``P dealias (N + f) = P dealias N + P dealias f``: the fused RHS without
forcing plus ``project(dealias(term))``.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import torch

from . import _native as nat
from .forcing import NoForcing, native_params
from .grid import _check_state, dealias_project

__all__ = ["NSParams", "make_ns_rhs", "linear_operator", "is_dealiased"]


@dataclass(frozen=True)
class NSParams:
    """Differentiable scalars of the RHS (navierstokes.py:40-59)."""

    nu: float
    forcing: object = field(default_factory=NoForcing)

    @property
    def label(self):
        return f"NavierStokes_nu{float(self.nu):g}_{self.forcing.label}"

    def __repr__(self):
        return f"NavierStokes(nu={float(self.nu):g}, forcing={self.forcing!r})"


def is_dealiased(u_hat, grid):
    """True when every mode outside the 2/3 box is exactly zero (then the
    transforms may skip those modes bit-for-bit).  One small reduction and a
    device->host read of one int."""
    flag = torch.empty(1, dtype=torch.int32, device=grid.device)
    nat.call("hit_check_dealiased", grid.plan.handle, nat.ptr(u_hat), nat.ptr(flag),
             nat.stream_ptr(grid.device))
    return int(flag.item()) == 0


def resolve_flags(u_hat, grid, assume_dealiased):
    if assume_dealiased is None:
        assume_dealiased = is_dealiased(u_hat, grid)
    return nat.HIT_FLAG_ASSUME_DEALIASED if assume_dealiased else 0


class NSRHS:
    """The callable returned by `make_ns_rhs` (navierstokes.py:62-97)."""

    def __init__(self, grid):
        self.grid = grid

    def __call__(self, u_hat, params, t, *, assume_dealiased=None, f_ext=None):
        """rhs(u_hat, params, t); ``f_ext`` (same layout as u_hat) is an
        external force added before the mask and the projection (no
        reference counterpart: the coarse-LES subgrid term)."""
        g = self.grid
        u_hat = _check_state(u_hat, g)
        flags = resolve_flags(u_hat, g, assume_dealiased)
        p = native_params(params.nu, params.forcing, flags)
        custom = p is None
        if custom:
            p = native_params(params.nu, NoForcing(), flags)
        du = torch.empty_like(u_hat)
        if f_ext is not None:
            f_ext = _check_state(f_ext, g)
            nat.call("hit_rhs_forced", g.plan.handle, nat.ptr(u_hat), p, nat.ptr(f_ext), float(t), nat.ptr(du),
                     nat.stream_ptr(g.device))
        else:
            nat.call("hit_rhs", g.plan.handle, nat.ptr(u_hat), p, float(t), nat.ptr(du),
                     nat.stream_ptr(g.device))
        if custom:
            du = du + dealias_project(params.forcing.term(u_hat, g, t) + torch.zeros_like(u_hat), g)
        return du

    def __repr__(self):
        return f"ns_rhs({self.grid!r})"


def make_ns_rhs(grid):
    """Build the RHS on `grid` (navierstokes.py:62-97)."""
    return NSRHS(grid)


def linear_operator(grid, params):
    """-nu k^2 (navierstokes.py:100-103)."""
    return -float(params.nu) * grid.k2
