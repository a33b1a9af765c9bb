"""Diagnostics (reference: src/hit3d/diagnostics.py).

The spectral reductions (E, Omega, eps, P, shell spectra) run in one fused
float64 kernel over the state (``hit_energy_budget`` / ``hit_energy_spectrum``);
scalar formulas stay on the host, as in the reference.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _native as nat
from .forcing import NoForcing, native_params
from .grid import _check_state, as_device, to_physical

__all__ = ["energy", "enstrophy", "dissipation", "energy_spectrum", "component_spectra",
           "compensated_spectrum", "dissipation_constant", "kolmogorov_scale",
           "taylor_microscale", "taylor_reynolds", "taylor_reynolds_field", "energy_budget",
           "energy_budget_cb", "velocity_samples", "velocity_moments",
           "longitudinal_autocorrelation", "integral_lengthscale"]


def _budget_raw(u_hat, grid, nu, forcing):
    """Device float64 [E, eps, P, Omega] of `u_hat`."""
    u_hat = _check_state(u_hat, grid)
    p = native_params(nu, forcing if forcing is not None else NoForcing())
    if p is None:
        p = native_params(nu, NoForcing())
    out = torch.empty(4, dtype=torch.float64, device=grid.device)
    nat.call("hit_energy_budget", grid.plan.handle, nat.ptr(u_hat), p, nat.ptr(out),
             nat.stream_ptr(grid.device))
    return out


def energy(u_hat, grid):
    """E = 1/2 <|u|^2> (diagnostics.py:56-58), float64 0-d device tensor."""
    return _budget_raw(u_hat, grid, 0.0, None)[0]


def enstrophy(u_hat, grid):
    """Omega = 1/2 <|w|^2> (diagnostics.py:61-65)."""
    return _budget_raw(u_hat, grid, 0.0, None)[3]


def dissipation(u_hat, grid, nu):
    """eps = 2 nu Omega (diagnostics.py:68-70)."""
    return _budget_raw(u_hat, grid, float(nu), None)[1]


def _spectra_dev(u_hat, grid):
    u_hat = _check_state(u_hat, grid)
    ns = grid.plan.num_shells
    E = torch.empty(ns, dtype=torch.float64, device=grid.device)
    Ec = torch.empty(3 * ns, dtype=torch.float64, device=grid.device)
    nat.call("hit_energy_spectrum", grid.plan.handle, nat.ptr(u_hat), nat.ptr(E), nat.ptr(Ec),
             nat.stream_ptr(grid.device))
    return E, Ec.view(3, ns)


def _ks(grid):
    k0 = 2 * np.pi / grid.Lx
    return np.arange(1, grid.num_shells + 1) * k0


def energy_spectrum(u_hat, grid):
    """Shell spectrum ``(k, E)`` as host arrays (diagnostics.py:94-101);
    E[s] is the energy of shell s+1, accumulated in float64."""
    E, _ = _spectra_dev(u_hat, grid)
    return _ks(grid), E.cpu().numpy()


def component_spectra(u_hat, grid):
    """``(k, E11, E22, E33)`` (diagnostics.py:104-114)."""
    _, Ec = _spectra_dev(u_hat, grid)
    Ec = Ec.cpu().numpy()
    return (_ks(grid), Ec[0], Ec[1], Ec[2])


def compensated_spectrum(ks, Es, eps, nu):
    """diagnostics.py:117-122."""
    eta = (nu**3 / eps) ** 0.25
    return ks * eta, Es * eps ** (-2 / 3) * ks ** (5 / 3)


def dissipation_constant(eps, ell, u_rms):
    """diagnostics.py:125-130."""
    return eps * ell / u_rms**3


def kolmogorov_scale(u_hat, grid, nu):
    """diagnostics.py:133-135."""
    return (nu**3 / float(dissipation(u_hat, grid, nu))) ** 0.25


def taylor_microscale(u_hat, grid):
    """diagnostics.py:138-140."""
    b = _budget_raw(u_hat, grid, 0.0, None)
    return float(np.sqrt(5 * float(b[0]) / float(b[3])))


def taylor_reynolds(E, eps, nu):
    """diagnostics.py:143-150."""
    u_p = np.sqrt(2 * E / 3)
    lam = np.sqrt(10 * nu * E / eps)
    return u_p * lam / nu


def taylor_reynolds_field(u_hat, grid, nu):
    """diagnostics.py:153-156."""
    b = _budget_raw(u_hat, grid, float(nu), None)
    return taylor_reynolds(float(b[0]), float(b[1]), nu)


def energy_budget(u_hat, grid, nu, forcing):
    """``{"E", "eps", "P"}`` (diagnostics.py:162-172) as float64 0-d device
    tensors; P is the forcing's exact injection."""
    b = _budget_raw(u_hat, grid, float(nu), forcing)
    if native_params(nu, forcing) is None:  # custom forcing: its own injection
        return {"E": b[0], "eps": b[1], "P": forcing.injection(u_hat, grid)}
    return {"E": b[0], "eps": b[1], "P": b[2]}


def energy_budget_cb(state):
    """Callback form of `energy_budget` (diagnostics.py:175-182)."""
    return energy_budget(state.u_hat, state.grid, state.params.nu, state.params.forcing)


def velocity_samples(u_hat, grid, component=0):
    """diagnostics.py:188-193."""
    u = to_physical(as_device(u_hat, grid, grid.cdtype)[component], grid)
    return u.cpu().numpy().ravel()


def velocity_moments(samples):
    """diagnostics.py:196-209."""
    samples = np.asarray(samples)
    m = samples.mean()
    c = samples - m
    v = np.mean(c**2)
    return {"mean": m, "variance": v, "skewness": np.mean(c**3) / v**1.5,
            "flatness": np.mean(c**4) / v**2}


def longitudinal_autocorrelation(u_hat, grid, component=0):
    """diagnostics.py:212-230 (Wiener-Khinchin through the CUDA c2r)."""
    u = as_device(u_hat, grid, grid.cdtype)[component]
    a2 = (u.real**2 + u.imag**2).to(grid.cdtype)
    ntot = grid.Nx * grid.Ny * grid.Nz
    corr = to_physical(a2, grid) / ntot
    n = grid.Nx // 2 + 1
    f = corr[:n, 0, 0].double().cpu().numpy()
    r = np.arange(n) * (grid.Lx / grid.Nx)
    if f[0] <= 0:
        return r, np.zeros_like(f)
    return r, f / f[0]


def integral_lengthscale(r, f):
    """diagnostics.py:233-244."""
    f = np.asarray(f)
    r = np.asarray(r)
    below = np.nonzero(f < 0)[0]
    n = (below[0] + 1) if below.size else len(f)
    if n < 2:
        return 0.0
    return float(np.trapezoid(f[:n], r[:n]))
