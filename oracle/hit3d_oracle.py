"""CPU oracle for the HIT3D pseudo-spectral Navier-Stokes hot path.

TEST INFRASTRUCTURE ONLY.  This module is a NumPy/SciPy restatement of the
reference package ``hit3d`` (nfrank22-gh/3DHIT, ``src/hit3d``).  It is the
checker for the CUDA implementation in ``3dhit_b200``: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` (its CPU-baseline leg and the
``--impl reference`` arm) may import it.  The product path never calls it.

Pinning.  The reference has no golden data files.  This restatement is pinned
(``tests/test_oracle_*.py``) by
  * the reference's own analytic known-answer tests (Beltrami decay, Parseval,
    projection, derivatives, injection exactness, budget residual), ported;
  * golden vectors produced by executing the reference's own source files
    (``grid.py``, ``forcing.py``, ``navierstokes.py``, ``integrators.py``,
    ``diagnostics.py``) on a NumPy-backed stand-in for ``jax.numpy``
    (``tests/golden/make_golden.py``).  jaxlib itself is not installable here,
    so the FFT underneath those vectors is numpy's pocketfft rather than
    jaxlib's ducc0 (same unnormalised-forward / 1/N inverse convention and the
    same irfftn axis order).

Precision follows the grid dtype exactly like the reference (float32 default,
float64 on request); NumPy 2 scalar promotion (NEP 50) matches JAX's weak
typing for Python scalars, so the operation dtypes are the reference's.
"""

from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np
import scipy.fft as sfft

_WORKERS = os.cpu_count() or 1


def set_workers(n):
    """Number of threads scipy.fft uses (the CPU baseline states it)."""
    global _WORKERS
    _WORKERS = max(1, int(n))


def get_workers():
    return _WORKERS


# ---------------------------------------------------------------------------
# grid.py  (reference: src/hit3d/grid.py)
# ---------------------------------------------------------------------------


@dataclass(frozen=True, eq=False)
class Grid:
    """Restates ``Grid`` (src/hit3d/grid.py:41-86)."""

    Nx: int
    Ny: int
    Nz: int
    Lx: float
    Ly: float
    Lz: float
    kx: np.ndarray
    ky: np.ndarray
    kz: np.ndarray
    k2: np.ndarray
    inv_k2: np.ndarray
    dealias: np.ndarray
    weights: np.ndarray

    @property
    def dtype(self):
        return self.k2.dtype

    @property
    def cdtype(self):
        return np.result_type(self.dtype, np.complex64)


def make_grid(Nx, Ny=None, Nz=None, *, Lx=2 * np.pi, Ly=2 * np.pi,
              Lz=2 * np.pi, dtype=np.float32):
    """``make_grid`` (src/hit3d/grid.py:89-132): wavenumbers computed in
    float64 then cast (:101-107), k2 in the run dtype (:109), inv_k2 with 0 at
    k=0 (:110-111), per-axis 2/3 box mask with k=0 removed (:115-120),
    Hermitian weights (:122-125)."""
    Ny = Nx if Ny is None else Ny
    Nz = Nx if Nz is None else Nz
    dtype = np.dtype(dtype)
    nx = np.fft.fftfreq(Nx, 1 / Nx)
    ny = np.fft.fftfreq(Ny, 1 / Ny)
    nz = np.arange(Nz // 2 + 1, dtype=float)
    kx = (2 * np.pi / Lx * nx).astype(dtype).reshape(-1, 1, 1)
    ky = (2 * np.pi / Ly * ny).astype(dtype).reshape(1, -1, 1)
    kz = (2 * np.pi / Lz * nz).astype(dtype).reshape(1, 1, -1)
    k2 = kx**2 + ky**2 + kz**2
    with np.errstate(divide="ignore"):
        inv_k2 = np.where(k2 == 0, dtype.type(0), 1 / k2).astype(dtype)
    mask = (
        (np.abs(nx).reshape(-1, 1, 1) <= Nx // 3)
        & (np.abs(ny).reshape(1, -1, 1) <= Ny // 3)
        & (np.abs(nz).reshape(1, 1, -1) <= Nz // 3)
    )
    mask[0, 0, 0] = False
    w = np.full(Nz // 2 + 1, 2, dtype=dtype)
    w[0] = 1
    if Nz % 2 == 0:
        w[-1] = 1
    return Grid(Nx=Nx, Ny=Ny, Nz=Nz, Lx=float(Lx), Ly=float(Ly), Lz=float(Lz),
                kx=kx, ky=ky, kz=kz, k2=k2, inv_k2=inv_k2, dealias=mask,
                weights=w.reshape(1, 1, -1))


def spectral_shape(grid):
    """src/hit3d/grid.py:135-137."""
    return (3, grid.Nx, grid.Ny, grid.Nz // 2 + 1)


def ddx(u_hat, grid):
    """src/hit3d/grid.py:146-148."""
    return 1j * grid.kx * u_hat


def ddy(u_hat, grid):
    """src/hit3d/grid.py:151-153."""
    return 1j * grid.ky * u_hat


def ddz(u_hat, grid):
    """src/hit3d/grid.py:156-158."""
    return 1j * grid.kz * u_hat


def laplacian(u_hat, grid):
    """src/hit3d/grid.py:161-163."""
    return -grid.k2 * u_hat


def dealias(u_hat, grid):
    """src/hit3d/grid.py:166-168 (multiplication by the boolean mask)."""
    return u_hat * grid.dealias


def project(u_hat, grid):
    """src/hit3d/grid.py:171-178, same operation order."""
    div = (grid.kx * u_hat[0] + grid.ky * u_hat[1] + grid.kz * u_hat[2]) \
        * grid.inv_k2
    return u_hat - np.stack((grid.kx * div, grid.ky * div, grid.kz * div))


def to_physical(u_hat, grid):
    """src/hit3d/grid.py:181-183: irfftn over the three spatial axes (complex
    inverse over x and y, c2r over z, 1/N per axis)."""
    return sfft.irfftn(u_hat, s=(grid.Nx, grid.Ny, grid.Nz), axes=(-3, -2, -1),
                       workers=_WORKERS)


def to_spectral(u, grid):
    """src/hit3d/grid.py:186-188: unnormalised rfftn over the spatial axes."""
    return sfft.rfftn(u, axes=(-3, -2, -1), workers=_WORKERS)


# ---------------------------------------------------------------------------
# forcing.py  (reference: src/hit3d/forcing.py)
# ---------------------------------------------------------------------------


def _ntot2(grid):
    """src/hit3d/forcing.py:44-45."""
    return np.asarray(grid.Nx * grid.Ny * grid.Nz, grid.dtype) ** 2


def _weighted_2E(u_hat, grid, mask=None):
    """src/hit3d/forcing.py:48-52."""
    w = grid.weights if mask is None else grid.weights * mask
    return np.sum(w * np.sum(np.abs(u_hat) ** 2, axis=0)) / _ntot2(grid)


@dataclass(frozen=True)
class NoForcing:
    """src/hit3d/forcing.py:55-71."""

    def term(self, u_hat, grid, t):
        return np.zeros((), dtype=u_hat.dtype)

    def injection(self, u_hat, grid):
        return np.zeros((), dtype=grid.dtype)

    @property
    def label(self):
        return "NoForcing"


@dataclass(frozen=True)
class LinearForcing:
    """Constant-coefficient Lundgren forcing f = A u
    (src/hit3d/forcing.py:74-106)."""

    A: float

    def term(self, u_hat, grid, t):
        return self.A * u_hat

    def injection(self, u_hat, grid):
        return self.A * _weighted_2E(u_hat, grid)

    @property
    def label(self):
        return f"LinearForcing_A{float(self.A):g}"


@dataclass(frozen=True)
class BandForcing:
    """Constant-power band forcing (src/hit3d/forcing.py:109-163)."""

    eps: float
    kmin: float
    kmax: float

    def _mask(self, grid):
        # src/hit3d/forcing.py:135-136
        return (self.kmin**2 <= grid.k2) & (grid.k2 <= self.kmax**2)

    def term(self, u_hat, grid, t):
        # src/hit3d/forcing.py:138-143
        mask = self._mask(grid)
        twoE = _weighted_2E(u_hat, grid, mask)
        tiny = np.finfo(grid.dtype).eps
        c = np.where(twoE > tiny, self.eps / np.where(twoE > tiny, twoE, 1), 0)
        c = np.asarray(c, grid.dtype)
        return c * mask * u_hat

    def injection(self, u_hat, grid):
        # src/hit3d/forcing.py:145-150
        twoE = _weighted_2E(u_hat, grid, self._mask(grid))
        tiny = np.finfo(grid.dtype).eps
        return np.asarray(np.where(twoE > tiny, self.eps, 0.0), grid.dtype)

    @property
    def label(self):
        return (f"BandForcing_eps{float(self.eps):g}"
                f"_k{float(self.kmin):g}-{float(self.kmax):g}")


@dataclass(frozen=True)
class HoldEnergyForcing:
    """Lundgren linear forcing whose coefficient holds a target kinetic energy
    (no reference counterpart; it follows the forcing contract of
    src/hit3d/forcing.py:8-20).

        A(u) = (eps - (E - E_target)/tau) / (2 E),   eps = 2 nu Omega,

    evaluated in float64 from the stage input's E and Omega; term = A u,
    injection = 2 A E.  tau = inf (the default) gives A = eps/(2E), which
    makes dE/dt = P - eps vanish identically in the semi-discrete system.
    ``nu`` must be the run's viscosity (the contract's ``term`` does not see
    the RHS parameters)."""

    E_target: float
    nu: float
    tau: float = math.inf

    def coefficient(self, u_hat, grid):
        E, Om = _energy_enstrophy_f64(u_hat, grid)
        if not E > 0:
            return 0.0
        relax = 0.0 if not np.isfinite(self.tau) else (E - self.E_target) / self.tau
        return (2.0 * self.nu * Om - relax) / (2.0 * E)

    def term(self, u_hat, grid, t):
        A = np.asarray(self.coefficient(u_hat, grid), grid.dtype)
        return A * u_hat

    def injection(self, u_hat, grid):
        E, _ = _energy_enstrophy_f64(u_hat, grid)
        return np.asarray(2.0 * self.coefficient(u_hat, grid) * E, grid.dtype)

    @property
    def label(self):
        return f"HoldEnergyForcing_E{float(self.E_target):g}"


def _energy_enstrophy_f64(u_hat, grid):
    """Hermitian-weighted Parseval sums in float64 (E, Omega)."""
    a2 = np.sum(np.abs(u_hat.astype(np.complex128)) ** 2, axis=0)
    w = grid.weights.astype(np.float64)
    n2 = float(grid.Nx * grid.Ny * grid.Nz) ** 2
    E = float(np.sum(w * a2) / n2 / 2)
    Om = float(np.sum(w * grid.k2.astype(np.float64) * a2) / n2 / 2)
    return E, Om


# ---------------------------------------------------------------------------
# navierstokes.py  (reference: src/hit3d/navierstokes.py)
# ---------------------------------------------------------------------------


@dataclass(frozen=True)
class NSParams:
    """src/hit3d/navierstokes.py:40-59."""

    nu: float
    forcing: object = field(default_factory=NoForcing)


def make_ns_rhs(grid):
    """src/hit3d/navierstokes.py:62-97: rotational form, forcing added before
    dealias+projection, viscous term last."""

    def rhs(u_hat, params, t):
        kx, ky, kz = grid.kx, grid.ky, grid.kz
        w_hat = 1j * np.stack((
            ky * u_hat[2] - kz * u_hat[1],
            kz * u_hat[0] - kx * u_hat[2],
            kx * u_hat[1] - ky * u_hat[0],
        ))
        u = to_physical(u_hat, grid)
        w = to_physical(w_hat, grid)
        nl = np.stack((
            u[1] * w[2] - u[2] * w[1],
            u[2] * w[0] - u[0] * w[2],
            u[0] * w[1] - u[1] * w[0],
        ))
        du = to_spectral(nl, grid) + params.forcing.term(u_hat, grid, t)
        du = project(dealias(du, grid), grid)
        return du - params.nu * grid.k2 * u_hat

    return rhs


def linear_operator(grid, params):
    """src/hit3d/navierstokes.py:100-103."""
    return -params.nu * grid.k2


# ---------------------------------------------------------------------------
# integrators.py  (reference: src/hit3d/integrators.py)
# ---------------------------------------------------------------------------


def rk4_step(rhs, u_hat, params, dt, t):
    """src/hit3d/integrators.py:32-38 (same stage inputs and combination
    order)."""
    k1 = rhs(u_hat, params, t)
    k2 = rhs(u_hat + 0.5 * dt * k1, params, t + 0.5 * dt)
    k3 = rhs(u_hat + 0.5 * dt * k2, params, t + 0.5 * dt)
    k4 = rhs(u_hat + dt * k3, params, t + dt)
    return u_hat + (dt / 6.0) * (k1 + 2 * k2 + 2 * k3 + k4)


def ifrk4_step(rhs, u_hat, params, dt, t, grid):
    """Integrating-factor (Lawson) RK4 on ``linear_operator``
    (src/hit3d/navierstokes.py:100-103), the scheme src/hit3d/integrators.py:15-16
    lists as to do; the reference has no implementation.  With
    E = exp(-nu k^2 dt/2) in the grid dtype and N the RHS at nu = 0 (the
    forcing keeps its own parameters):

        k1 = N(u), k2 = N(E (u + dt/2 k1)), k3 = N(E u + dt/2 k2),
        k4 = N(E^2 u + dt E k3),
        u' = E^2 u + dt/6 ((E (E k1 + 2 k2) + 2 E k3) + k4)

    (the grouping the fused CUDA epilogue uses)."""
    rt = grid.dtype.type
    E = np.exp(rt(-0.5 * dt * params.nu) * grid.k2).astype(grid.dtype)
    p0 = NSParams(nu=0.0, forcing=params.forcing)
    k1 = rhs(u_hat, p0, t)
    k2 = rhs(E * (u_hat + 0.5 * dt * k1), p0, t + 0.5 * dt)
    k3 = rhs(E * u_hat + 0.5 * dt * k2, p0, t + 0.5 * dt)
    ek3 = E * k3
    k4 = rhs((E * E) * u_hat + dt * ek3, p0, t + dt)
    return (E * E) * u_hat + (dt / 6.0) * ((E * (E * k1 + 2 * k2) + 2 * ek3) + k4)


def rollout(rhs, u_hat, params, dt, nsteps, t0=0.0, callback=None):
    """src/hit3d/integrators.py:41-53 (the scan body as a loop).  The
    optional ``callback(step, u_hat)`` is an oracle-only hook used by tests
    to sample states along the way."""
    for i in range(nsteps):
        u_hat = rk4_step(rhs, u_hat, params, dt, t0 + i * dt)
        if callback is not None:
            callback(i + 1, u_hat)
    return u_hat


# ---------------------------------------------------------------------------
# diagnostics.py  (reference: src/hit3d/diagnostics.py)
# ---------------------------------------------------------------------------


def _norm2(grid):
    """src/hit3d/diagnostics.py:45-46."""
    return np.asarray(grid.Nx * grid.Ny * grid.Nz, grid.dtype) ** 2


def _weighted_sum(a2, grid, extra=None):
    """src/hit3d/diagnostics.py:49-53."""
    w = grid.weights if extra is None else grid.weights * extra
    return np.sum(w * a2) / _norm2(grid)


def energy(u_hat, grid):
    """src/hit3d/diagnostics.py:56-58."""
    return _weighted_sum(np.sum(np.abs(u_hat) ** 2, axis=0), grid) / 2


def enstrophy(u_hat, grid):
    """src/hit3d/diagnostics.py:61-65."""
    return _weighted_sum(np.sum(np.abs(u_hat) ** 2, axis=0), grid,
                         extra=grid.k2) / 2


def dissipation(u_hat, grid, nu):
    """src/hit3d/diagnostics.py:68-70."""
    return 2 * nu * enstrophy(u_hat, grid)


def shells(grid):
    """src/hit3d/diagnostics.py:76-82: shell = floor(sqrt(k2)/k0 + 0.5) in the
    grid dtype, smax = ceil(sqrt(3) max(N)/2) + 1."""
    k0 = 2 * np.pi / grid.Lx
    smax = int(np.ceil(np.sqrt(3) * max(grid.Nx, grid.Ny, grid.Nz) / 2)) + 1
    shell = np.floor(np.sqrt(grid.k2) / k0 + 0.5).astype(np.int32)
    return shell, smax, k0


def _shell_sum(a2, grid):
    """src/hit3d/diagnostics.py:85-91 (bincount, bin 0 dropped)."""
    shell, smax, _ = shells(grid)
    e = (grid.weights * a2) / (2 * _norm2(grid))
    out = np.bincount(shell.ravel(), weights=e.ravel(), minlength=smax + 1)
    return out[: smax + 1].astype(grid.dtype)[1:]


def energy_spectrum(u_hat, grid):
    """src/hit3d/diagnostics.py:94-101."""
    _, smax, k0 = shells(grid)
    ks = np.arange(1, smax + 1) * k0
    return ks, _shell_sum(np.sum(np.abs(u_hat) ** 2, axis=0), grid)


def component_spectra(u_hat, grid):
    """src/hit3d/diagnostics.py:104-114."""
    _, smax, k0 = shells(grid)
    ks = np.arange(1, smax + 1) * k0
    return (ks, *[_shell_sum(np.abs(u_hat[i]) ** 2, grid) for i in range(3)])


def energy_spectrum_f64(u_hat, grid):
    """Float64-accumulated counterpart of ``energy_spectrum`` (the CUDA
    diagnostics accumulate in float64); shells as in the reference."""
    shell, smax, k0 = shells(grid)
    a2 = np.abs(u_hat.astype(np.complex128)) ** 2
    e = grid.weights.astype(np.float64) * a2 / (2 * float(grid.Nx * grid.Ny * grid.Nz) ** 2)
    comp = [np.bincount(shell.ravel(), weights=e[c].ravel(),
                        minlength=smax + 1)[: smax + 1][1:] for c in range(3)]
    return np.arange(1, smax + 1) * k0, comp[0] + comp[1] + comp[2], comp


def energy_budget(u_hat, grid, nu, forcing):
    """src/hit3d/diagnostics.py:162-172."""
    return {"E": energy(u_hat, grid), "eps": dissipation(u_hat, grid, nu),
            "P": forcing.injection(u_hat, grid)}


def energy_budget_f64(u_hat, grid, nu, forcing):
    """Float64-accumulated budget (what the CUDA kernels compute)."""
    E, Om = _energy_enstrophy_f64(u_hat, grid)
    if isinstance(forcing, NoForcing):
        P = 0.0
    elif isinstance(forcing, LinearForcing):
        P = float(forcing.A) * 2 * E
    elif isinstance(forcing, BandForcing):
        m = forcing._mask(grid)
        a2 = np.sum(np.abs(u_hat.astype(np.complex128)) ** 2, axis=0)
        twoE = float(np.sum(grid.weights.astype(np.float64) * m * a2)) \
            / float(grid.Nx * grid.Ny * grid.Nz) ** 2
        P = float(forcing.eps) if twoE > np.finfo(grid.dtype).eps else 0.0
    elif isinstance(forcing, HoldEnergyForcing):
        P = 2 * forcing.coefficient(u_hat, grid) * E
    else:
        raise TypeError(forcing)
    return {"E": E, "eps": 2 * nu * Om, "P": P}


# ---------------------------------------------------------------------------
# fields.py  (reference: src/hit3d/fields.py) -- seeds via NumPy PCG64
# ---------------------------------------------------------------------------


def spectral_state(grid):
    """src/hit3d/fields.py:39-41."""
    return np.zeros(spectral_shape(grid), dtype=grid.cdtype)


def default_spectrum(k):
    """src/hit3d/fields.py:30-32."""
    return k**4 * np.exp(-2 * k**2)


def rm_spectrum(u0=1.0, k0=4.0):
    """Rosales-Meneveau Eq. 9, as the reference drivers write it
    (scripts/generate_dataset.py:87-92)."""
    return lambda k: (16 * np.sqrt(2 / np.pi) * u0**2 / k0**5
                      * k**4 * np.exp(-2 * k**2 / k0**2))


def white_noise(seed, grid):
    """Uniform white noise in [-0.5, 0.5) from NumPy's PCG64 (stands in for
    jax.random.uniform at src/hit3d/fields.py:45-46)."""
    rng = np.random.default_rng(seed)
    return rng.random((3, grid.Nx, grid.Ny, grid.Nz), dtype=grid.dtype) \
        - grid.dtype.type(0.5)


def shell_rescale(u_hat, grid, spectrum):
    """src/hit3d/fields.py:51-68: per-shell rescale to the target spectrum."""
    k0 = 2 * np.pi / grid.Lx
    smax = int(np.ceil(np.sqrt(3) * max(grid.Nx, grid.Ny, grid.Nz) / 2)) + 1
    shell = np.floor(np.sqrt(grid.k2) / k0 + 0.5).astype(np.int32)
    ntot2 = np.asarray(grid.Nx * grid.Ny * grid.Nz, grid.dtype) ** 2
    e_mode = grid.weights * np.sum(np.abs(u_hat) ** 2, axis=0) / (2 * ntot2)
    Es = np.bincount(shell.ravel(), weights=e_mode.ravel(),
                     minlength=smax + 1)[: smax + 1].astype(grid.dtype)
    ks = np.arange(smax + 1, dtype=grid.dtype) * k0
    target = spectrum(ks)
    Es_safe = np.where(Es > 0, Es, 1)
    with np.errstate(invalid="ignore", divide="ignore"):
        c = np.where(Es > 0, np.where(target > 0, np.sqrt(target / Es_safe), 0.0),
                     1.0).astype(grid.dtype)
    return u_hat * c[shell]


def random_field(seed, grid, spectrum=default_spectrum):
    """src/hit3d/fields.py:35-68 with a PCG64 seed."""
    u = white_noise(seed, grid)
    u_hat = project(dealias(to_spectral(u, grid), grid), grid)
    return shell_rescale(u_hat, grid, spectrum)


def hit_initial_field(seed, grid, u0=1.0, k0=4.0, E_target=1.5):
    """The benchmark initial condition: random_field with the RM Eq. 9
    spectrum, then one global rescale to E = E_target (u_rms = 1)."""
    u_hat = random_field(seed, grid, rm_spectrum(u0, k0))
    E, _ = _energy_enstrophy_f64(u_hat, grid)
    return (u_hat * np.asarray(np.sqrt(E_target / E), grid.dtype)).astype(grid.cdtype)


def taylor_green(grid):
    """src/hit3d/fields.py:71-87."""
    t = grid.dtype
    x = (np.arange(grid.Nx, dtype=t) * t.type(2 * np.pi / grid.Nx)).reshape(-1, 1, 1)
    y = (np.arange(grid.Ny, dtype=t) * t.type(2 * np.pi / grid.Ny)).reshape(1, -1, 1)
    z = (np.arange(grid.Nz, dtype=t) * t.type(2 * np.pi / grid.Nz)).reshape(1, 1, -1)
    u = np.stack((
        np.sin(x) * np.cos(y) * np.cos(z),
        -np.cos(x) * np.sin(y) * np.cos(z),
        np.zeros((grid.Nx, grid.Ny, grid.Nz), dtype=t),
    ))
    return dealias(to_spectral(u, grid), grid)


def beltrami(grid):
    """ABC flow used by the reference tests (tests/conftest.py:16-30)."""
    t = grid.dtype
    x = (np.arange(grid.Nx, dtype=t) * t.type(2 * np.pi / grid.Nx)).reshape(-1, 1, 1)
    y = (np.arange(grid.Ny, dtype=t) * t.type(2 * np.pi / grid.Ny)).reshape(1, -1, 1)
    z = (np.arange(grid.Nz, dtype=t) * t.type(2 * np.pi / grid.Nz)).reshape(1, 1, -1)
    shape = (grid.Nx, grid.Ny, grid.Nz)
    u = np.stack((
        np.broadcast_to(np.sin(z) + np.cos(y), shape),
        np.broadcast_to(np.sin(x) + np.cos(z), shape),
        np.broadcast_to(np.sin(y) + np.cos(x), shape),
    ))
    return to_spectral(u, grid)


# ---------------------------------------------------------------------------
# CFL time step (no reference counterpart; the reference takes dt as input)
# ---------------------------------------------------------------------------


def cfl_dt(u_hat, grid, cfl=0.5):
    """dt = cfl * dx / max_x(|u|+|v|+|w|), dx = min(L_i/N_i), computed in
    float64 from the physical field of ``u_hat``."""
    u = to_physical(u_hat, grid).astype(np.float64)
    umax = float(np.max(np.abs(u[0]) + np.abs(u[1]) + np.abs(u[2])))
    dx = min(grid.Lx / grid.Nx, grid.Ly / grid.Ny, grid.Lz / grid.Nz)
    return cfl * dx / umax


# ---------------------------------------------------------------------------
# Discrete adjoint (no reference counterpart: the reference differentiates
# through jax.vjp of src/hit3d/navierstokes.py:62-97 and
# src/hit3d/integrators.py:32-53).  A cotangent is dL/dRe + i dL/dIm of the
# stored half-spectrum entries, i.e. the inner product is
# <a, b> = sum Re(conj(a) b) over the stored array; the transpose of a
# complex-linear operator is then its conjugate transpose.  jax.vjp returns
# the complex conjugate of these cotangents.
# ---------------------------------------------------------------------------


def _cross(a, b):
    return np.stack((a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]))


def _curl_hat(u_hat, grid):
    """1j k x u_hat (navierstokes.py:73-77); its own transpose."""
    kx, ky, kz = grid.kx, grid.ky, grid.kz
    return 1j * np.stack((ky * u_hat[2] - kz * u_hat[1], kz * u_hat[0] - kx * u_hat[2], kx * u_hat[1] - ky * u_hat[0]))


def _dot_re(a, b, extra=None):
    """sum Re(conj(a) b) in float64 (optionally weighted per mode)."""
    p = np.real(np.conj(a.astype(np.complex128)) * b.astype(np.complex128))
    if extra is not None:
        p = p * extra
    return float(np.sum(p))


def to_physical_T(v, grid):
    """Transpose of to_physical: w rfftn(v) / N^3 (w = Hermitian weights)."""
    n3 = grid.Nx * grid.Ny * grid.Nz
    return (grid.weights * to_spectral(v, grid) / n3).astype(grid.cdtype)


def to_spectral_T(v_hat, grid):
    """Transpose of to_spectral: N^3 irfftn(v_hat / w)."""
    n3 = grid.Nx * grid.Ny * grid.Nz
    return (n3 * to_physical(v_hat / grid.weights, grid)).astype(grid.dtype)


def forcing_vjp(forcing, u_hat, grid, pv):
    """Transpose of the derivative of ``forcing.term`` at u_hat applied to pv:
    (u_hat cotangent, {parameter: cotangent}) (forcing.py:94-95, 138-143 and
    the hold-energy coefficient)."""
    ntot2 = float(grid.Nx * grid.Ny * grid.Nz) ** 2
    w = grid.weights.astype(np.float64)
    if isinstance(forcing, LinearForcing):
        return forcing.A * pv, {"A": _dot_re(pv, u_hat)}
    if isinstance(forcing, BandForcing):
        mask = forcing._mask(grid)
        twoE = float(_weighted_2E(u_hat, grid, mask))
        if not twoE > float(np.finfo(grid.dtype).eps):
            return np.zeros_like(pv), {"eps": 0.0}
        c = forcing.eps / twoE
        beta = _dot_re(pv, u_hat, mask)
        # c = eps / 2E_band,  d(2E_band)/du = 2 w mask u / Ntot^2
        ub = c * mask * pv + (beta * (-c / twoE) * 2.0 / ntot2) * (w * mask * u_hat)
        return ub.astype(grid.cdtype), {"eps": beta / twoE}
    if isinstance(forcing, HoldEnergyForcing):
        E, Om = _energy_enstrophy_f64(u_hat, grid)
        if not E > 0:
            return np.zeros_like(pv), {"nu": 0.0}
        A = forcing.coefficient(u_hat, grid)
        itau = 0.0 if not np.isfinite(forcing.tau) else 1.0 / forcing.tau
        beta = _dot_re(pv, u_hat)
        dA_dE = -itau / (2.0 * E) - A / E
        dA_dO = forcing.nu / E
        k2 = grid.k2.astype(np.float64)
        ub = A * pv + (beta / ntot2) * (dA_dE * w + dA_dO * w * k2) * u_hat
        return ub.astype(grid.cdtype), {"nu": beta * Om / E}
    return np.zeros_like(pv), {}


def rhs_vjp(grid, u_hat, params, v):
    """Transpose of the RHS derivative at u_hat applied to the cotangent v of
    rhs(u_hat): returns (u_hat cotangent, {"nu", "A", "eps": cotangents}).

    With g = irfftn(pv / w), pv = project(dealias(v)), u = irfftn(u_hat) and
    w_ = irfftn(1j k x u_hat), the nonlinear term contributes
    w (rfftn(w_ x g) + 1j k x rfftn(g x u)); the viscous term -nu k2 v; the
    forcing term forcing_vjp(pv)."""
    u_hat = np.asarray(u_hat, grid.cdtype)
    v = np.asarray(v, grid.cdtype)
    pv = project(dealias(v, grid), grid)
    pbar = {"nu": -_dot_re(v, u_hat, grid.k2.astype(np.float64)), "A": 0.0, "eps": 0.0}
    fb, fp = forcing_vjp(params.forcing, u_hat, grid, pv)
    for k, val in fp.items():
        pbar[k] += val
    u = to_physical(u_hat, grid)
    om = to_physical(_curl_hat(u_hat, grid), grid)
    g = to_physical(pv / grid.weights, grid)
    nl_bar = grid.weights * (to_spectral(_cross(om, g), grid) + _curl_hat(to_spectral(_cross(g, u), grid), grid))
    ub = nl_bar.astype(grid.cdtype) - params.nu * grid.k2 * v + fb
    return ub.astype(grid.cdtype), pbar


def _add_params(a, b):
    return {k: a.get(k, 0.0) + b.get(k, 0.0) for k in set(a) | set(b)}


def rk4_step_vjp(grid, u_hat, params, dt, ub, t=0.0):
    """Transpose of rk4_step (integrators.py:32-38) at u_hat applied to the
    cotangent ub of the new state; the stage inputs are recomputed."""
    rhs = make_ns_rhs(grid)
    u_hat = np.asarray(u_hat, grid.cdtype)
    ub = np.asarray(ub, grid.cdtype)
    k1 = rhs(u_hat, params, t)
    s2 = u_hat + 0.5 * dt * k1
    k2 = rhs(s2, params, t + 0.5 * dt)
    s3 = u_hat + 0.5 * dt * k2
    k3 = rhs(s3, params, t + 0.5 * dt)
    s4 = u_hat + dt * k3
    sb4, p4 = rhs_vjp(grid, s4, params, (dt / 6.0) * ub)
    sb3, p3 = rhs_vjp(grid, s3, params, (dt / 3.0) * ub + dt * sb4)
    sb2, p2 = rhs_vjp(grid, s2, params, (dt / 3.0) * ub + 0.5 * dt * sb3)
    sb1, p1 = rhs_vjp(grid, u_hat, params, (dt / 6.0) * ub + 0.5 * dt * sb2)
    pbar = _add_params(_add_params(p1, p2), _add_params(p3, p4))
    return (ub + sb1 + sb2 + sb3 + sb4).astype(grid.cdtype), pbar


def rollout_vjp(grid, u0, params, dt, nsteps, ub, t0=0.0, checkpoint_every=None):
    """Transpose of rollout (integrators.py:41-53): states are kept every
    ``checkpoint_every`` steps and recomputed segment by segment."""
    K = nsteps if not checkpoint_every else int(checkpoint_every)
    rhs = make_ns_rhs(grid)
    ckpt = []
    u = np.asarray(u0, grid.cdtype)
    for i in range(nsteps):
        if i % K == 0:
            ckpt.append(u)
        u = rk4_step(rhs, u, params, dt, t0 + i * dt)
    ub = np.asarray(ub, grid.cdtype)
    pbar = {"nu": 0.0, "A": 0.0, "eps": 0.0}
    for j in range(len(ckpt) - 1, -1, -1):
        i0 = j * K
        seg = [ckpt[j]]
        for i in range(i0, min(i0 + K, nsteps) - 1):
            seg.append(rk4_step(rhs, seg[-1], params, dt, t0 + i * dt))
        for i in range(len(seg) - 1, -1, -1):
            ub, p = rk4_step_vjp(grid, seg[i], params, dt, ub, t0 + (i0 + i) * dt)
            pbar = _add_params(pbar, p)
    return ub, pbar


# ---------------------------------------------------------------------------
# Learned SGS closure MLP (no reference counterpart): 9 -> 64 -> 64 -> 64 -> 6,
# GELU (tanh form), restated with the tensor-core kernels' bf16 roundings (bf16
# weights, inputs, hidden activations and backward gradients; float32 biases
# and pre-activations; sums in float64), so the CUDA forward, loss and weight
# gradients can be checked against it.
# ---------------------------------------------------------------------------


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even), as float32."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    b = a.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16 << 16
    return b.astype(np.uint32).view(np.float32).reshape(a.shape)


_S2PI = np.sqrt(2.0 / np.pi)


def _gelu(x):
    """GELU, tanh form (Hendrycks and Gimpel, 2016), the kernels' activation."""
    t = np.tanh(_S2PI * (x + 0.044715 * x ** 3))
    return 0.5 * x * (1.0 + t)


def _gelu_d(x):
    t = np.tanh(_S2PI * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * _S2PI * (1.0 + 3 * 0.044715 * x * x)


def mlp_loss_grads(params, x, tau):
    """params = (W1 [9,64], b1, W2 [64,64], b2, W3, b3, W4 [64,6], b4) float32;
    x [P,9], tau [P,6].  Returns (y, loss, grads) with grads in the params'
    order; loss = mean((y - tau)^2)."""
    W1, b1, W2, b2, W3, b3, W4, b4 = [np.asarray(p, np.float32) for p in params]
    P = x.shape[0]
    f64 = np.float64
    a0 = bf16(x).astype(f64)
    z1 = a0 @ bf16(W1).astype(f64) + bf16(b1).astype(f64)
    a1 = bf16(_gelu(z1.astype(np.float32))).astype(f64)
    z2 = a1 @ bf16(W2).astype(f64) + b2
    a2 = bf16(_gelu(z2.astype(np.float32))).astype(f64)
    z3 = a2 @ bf16(W3).astype(f64) + b3
    a3 = bf16(_gelu(z3.astype(np.float32))).astype(f64)
    y = a3 @ bf16(W4).astype(f64) + b4
    r = y - tau
    loss = float(np.mean(r * r))
    dz4 = bf16((2.0 * r / (P * 6)).astype(np.float32)).astype(f64)
    da3 = dz4 @ bf16(W4).astype(f64).T
    dz3 = bf16((da3 * _gelu_d(z3)).astype(np.float32)).astype(f64)
    da2 = dz3 @ bf16(W3).astype(f64).T
    dz2 = bf16((da2 * _gelu_d(z2)).astype(np.float32)).astype(f64)
    da1 = dz2 @ bf16(W2).astype(f64).T
    dz1 = bf16((da1 * _gelu_d(z1)).astype(np.float32)).astype(f64)
    grads = (a0.T @ dz1, dz1.sum(0), a1.T @ dz2, dz2.sum(0), a2.T @ dz3, dz3.sum(0), a3.T @ dz4, dz4.sum(0))
    return y, loss, grads
