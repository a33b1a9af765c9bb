"""Initial conditions (reference: src/hit3d/fields.py) and the CFL step.

`random_field` runs on the device: uniform noise (torch Philox generator,
or NumPy PCG64 with ``host_noise=True`` to reproduce the CPU oracle's noise)
-> rfftn -> dealias -> project -> per-shell rescale, the reference's route
(fields.py:35-68) through this package's own kernels.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _native as nat
from .diagnostics import _budget_raw, _spectra_dev
from .grid import as_device, dealias, dealias_project, spectral_shape, to_physical, to_spectral

__all__ = ["spectral_state", "random_field", "taylor_green", "default_spectrum", "rm_spectrum",
           "hit_initial_field", "cfl_dt"]


def spectral_state(grid):
    """Zero state (fields.py:39-41)."""
    return torch.zeros(spectral_shape(grid), dtype=grid.cdtype, device=grid.device)


def default_spectrum(k):
    """k^4 exp(-2 k^2) (fields.py:30-32); numpy or torch input."""
    lib = torch if isinstance(k, torch.Tensor) else np
    return k**4 * lib.exp(-2 * k**2)


def rm_spectrum(u0=1.0, k0=4.0):
    """Rosales-Meneveau Eq. 9, as the reference drivers use it
    (scripts/generate_dataset.py:87-92)."""
    def spec(k):
        lib = torch if isinstance(k, torch.Tensor) else np
        return 16 * np.sqrt(2 / np.pi) * u0**2 / k0**5 * k**4 * lib.exp(-2 * k**2 / k0**2)
    return spec


def _noise(seed, grid, host_noise):
    shape = (3, grid.Nx, grid.Ny, grid.Nz)
    if host_noise:
        rng = np.random.default_rng(seed)
        npdt = np.float32 if grid.dtype == torch.float32 else np.float64
        u = rng.random(shape, dtype=npdt) - npdt(0.5)
        return as_device(u, grid, grid.dtype)
    gen = torch.Generator(device=grid.device)
    gen.manual_seed(int(seed))
    return torch.rand(shape, generator=gen, dtype=grid.dtype, device=grid.device) - 0.5


def random_field(seed, grid, spectrum=default_spectrum, *, host_noise=False):
    """Solenoidal random field whose shell spectrum matches ``spectrum(k)``
    (fields.py:35-68)."""
    u_hat = dealias_project(to_spectral(_noise(seed, grid, host_noise), grid), grid)
    E, _ = _spectra_dev(u_hat, grid)          # shells 1..smax, float64
    Es = np.concatenate([[0.0], E.cpu().numpy()])  # shell 0 holds only k = 0 (masked)
    k0 = 2 * np.pi / grid.Lx
    ks = np.arange(grid.num_shells + 1) * k0
    target = np.asarray(spectrum(ks), dtype=np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        c = np.where(Es > 0, np.where(target > 0, np.sqrt(target / np.where(Es > 0, Es, 1)), 0.0), 1.0)
    c_dev = torch.from_numpy(c).to(grid.device)
    out = torch.empty_like(u_hat)
    nat.call("hit_shell_scale", grid.plan.handle, nat.ptr(u_hat), nat.ptr(c_dev), nat.ptr(out),
             nat.stream_ptr(grid.device))
    return out


def hit_initial_field(seed, grid, u0=1.0, k0=4.0, E_target=1.5, *, host_noise=False):
    """Benchmark initial condition: random_field with the RM Eq. 9 spectrum,
    then one global rescale to E = E_target (u_rms = 1 for 1.5)."""
    u = random_field(seed, grid, rm_spectrum(u0, k0), host_noise=host_noise)
    E = float(_budget_raw(u, grid, 0.0, None)[0])
    return u * float(np.sqrt(E_target / E))


def taylor_green(grid):
    """Taylor-Green vortex (fields.py:71-87)."""
    t = grid.dtype
    dev = grid.device
    x = (torch.arange(grid.Nx, dtype=t, device=dev) * (2 * np.pi / grid.Nx)).reshape(-1, 1, 1)
    y = (torch.arange(grid.Ny, dtype=t, device=dev) * (2 * np.pi / grid.Ny)).reshape(1, -1, 1)
    z = (torch.arange(grid.Nz, dtype=t, device=dev) * (2 * np.pi / grid.Nz)).reshape(1, 1, -1)
    u = torch.stack((torch.sin(x) * torch.cos(y) * torch.cos(z),
                     -torch.cos(x) * torch.sin(y) * torch.cos(z),
                     torch.zeros((grid.Nx, grid.Ny, grid.Nz), dtype=t, device=dev)))
    return dealias(to_spectral(u, grid), grid)


def cfl_dt(u_hat, grid, cfl=0.5):
    """dt = cfl * dx / max(|u|+|v|+|w|) from the physical field (no reference
    counterpart; the reference takes dt as an input)."""
    u = to_physical(as_device(u_hat, grid, grid.cdtype), grid)
    umax = float((u[0].abs() + u[1].abs() + u[2].abs()).max())
    dx = min(grid.Lx / grid.Nx, grid.Ly / grid.Ny, grid.Lz / grid.Nz)
    return cfl * dx / umax
