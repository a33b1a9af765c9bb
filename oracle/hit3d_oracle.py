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
