"""Forcing plug-ins (reference: src/hit3d/forcing.py).

Same contract as the reference (forcing.py:8-20): ``term(u_hat, grid, t)``,
``injection(u_hat, grid)`` and ``label``.  The fused RHS kernel implements
each built-in forcing itself (``native()`` gives its C-ABI parameters); the
``term`` methods exist for callers of the plug-in API and for custom
forcings, which the RHS adds through ``project(dealias(term))``.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import torch

from . import _native as nat

__all__ = ["NoForcing", "LinearForcing", "BandForcing", "HoldEnergyForcing"]


def _fmt(x):
    return f"{float(x):g}"


def _tiny(grid):
    return torch.finfo(grid.dtype).eps


def _weighted_2E(u_hat, grid, mask=None):
    """2E with Hermitian weights (forcing.py:48-52), accumulated in float64."""
    a2 = (u_hat.real.double() ** 2 + u_hat.imag.double() ** 2).sum(0)
    w = grid.weights.double()
    if mask is not None:
        w = w * mask
    n2 = float(grid.Nx * grid.Ny * grid.Nz) ** 2
    return (w * a2).sum() / n2


@dataclass(frozen=True)
class NoForcing:
    """Decaying turbulence (forcing.py:55-71)."""

    def term(self, u_hat, grid, t):
        return torch.zeros((), dtype=grid.cdtype, device=grid.device)

    def injection(self, u_hat, grid):
        from .diagnostics import energy_budget
        return energy_budget(u_hat, grid, 0.0, self)["P"]

    def native(self):
        return dict(forcing_kind=nat.HIT_FORCING_NONE)

    @property
    def label(self):
        return "NoForcing"

    def __repr__(self):
        return "NoForcing()"


@dataclass(frozen=True)
class LinearForcing:
    """Lundgren's linear forcing f = A u with constant A (forcing.py:74-106)."""

    A: float

    def term(self, u_hat, grid, t):
        return float(self.A) * u_hat

    def injection(self, u_hat, grid):
        """P = 2 A E (forcing.py:97-99)."""
        from .diagnostics import energy_budget
        return energy_budget(u_hat, grid, 0.0, self)["P"]

    def native(self):
        return dict(forcing_kind=nat.HIT_FORCING_LINEAR, A=float(self.A))

    @property
    def label(self):
        return f"LinearForcing_A{_fmt(self.A)}"

    def __repr__(self):
        return f"LinearForcing(A={_fmt(self.A)})"


@dataclass(frozen=True)
class BandForcing:
    """Constant-power forcing on kmin <= |k| <= kmax: f = eps/(2 E_band) u on
    the band, zero if the band holds no energy (forcing.py:109-163)."""

    eps: float
    kmin: float
    kmax: float

    def _mask(self, grid):
        return (float(self.kmin) ** 2 <= grid.k2) & (grid.k2 <= float(self.kmax) ** 2)

    def term(self, u_hat, grid, t):
        mask = self._mask(grid)
        twoE = float(_weighted_2E(u_hat, grid, mask))
        c = float(self.eps) / twoE if twoE > _tiny(grid) else 0.0
        return (c * mask.to(grid.dtype)) * u_hat

    def injection(self, u_hat, grid):
        """``eps`` when the band holds energy, else 0 (forcing.py:145-150)."""
        from .diagnostics import energy_budget
        return energy_budget(u_hat, grid, 0.0, self)["P"]

    def native(self):
        return dict(forcing_kind=nat.HIT_FORCING_BAND, eps=float(self.eps),
                    kmin=float(self.kmin), kmax=float(self.kmax))

    @property
    def label(self):
        return f"BandForcing_eps{_fmt(self.eps)}_k{_fmt(self.kmin)}-{_fmt(self.kmax)}"

    def __repr__(self):
        return f"BandForcing(eps={_fmt(self.eps)}, k=[{_fmt(self.kmin)}, {_fmt(self.kmax)}])"


@dataclass(frozen=True)
class HoldEnergyForcing:
    """Lundgren linear forcing whose coefficient holds the kinetic energy at
    ``E_target`` (no reference counterpart; same plug-in contract):

        A = (2 nu Omega - (E - E_target)/tau) / (2 E),  term = A u,  P = 2 A E,

    with E and Omega of the RHS input, evaluated in float64 on the GPU inside
    every RHS.  ``tau = inf`` (default) makes dE/dt = P - eps vanish exactly in
    the semi-discrete system.  ``nu`` must be the run's viscosity."""

    E_target: float
    nu: float
    tau: float = math.inf

    def coefficient(self, u_hat, grid):
        from .diagnostics import _budget_raw
        b = _budget_raw(u_hat, grid, float(self.nu), self)
        E, Om = float(b[0]), float(b[3])
        if not E > 0:
            return 0.0
        relax = (E - float(self.E_target)) / float(self.tau) if math.isfinite(self.tau) and self.tau > 0 else 0.0
        return (2.0 * float(self.nu) * Om - relax) / (2.0 * E)

    def term(self, u_hat, grid, t):
        return self.coefficient(u_hat, grid) * u_hat

    def injection(self, u_hat, grid):
        from .diagnostics import energy_budget
        return energy_budget(u_hat, grid, float(self.nu), self)["P"]

    def native(self):
        tau = float(self.tau)
        return dict(forcing_kind=nat.HIT_FORCING_HOLD_ENERGY, E_target=float(self.E_target),
                    tau=tau if math.isfinite(tau) else 0.0)

    @property
    def label(self):
        return f"HoldEnergyForcing_E{_fmt(self.E_target)}"

    def __repr__(self):
        return f"HoldEnergyForcing(E_target={_fmt(self.E_target)}, tau={_fmt(self.tau)})"


BUILTIN = (NoForcing, LinearForcing, BandForcing, HoldEnergyForcing)


def native_params(nu, forcing, flags=0):
    """HitParams for a built-in forcing (None for a custom one)."""
    if not isinstance(forcing, BUILTIN):
        return None
    kw = dict(nu=float(nu), flags=int(flags), forcing_kind=0, A=0.0, eps=0.0, kmin=0.0, kmax=0.0,
              E_target=0.0, tau=0.0)
    kw.update(forcing.native())
    if isinstance(forcing, HoldEnergyForcing) and float(forcing.nu) != float(nu):
        raise ValueError(f"HoldEnergyForcing.nu={forcing.nu} differs from NSParams.nu={nu}")
    return nat.HitParams(**kw)
