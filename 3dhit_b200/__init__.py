"""B200-native HIT3D: the pseudo-spectral Navier-Stokes step, rollout,
forcings and spectral diagnostics of nfrank22-gh/3DHIT (package ``hit3d``)
as hand-written sm_100a CUDA kernels behind a C ABI (include/hit3d.h).

Same pure-function API over the complex state ``(3, Nx, Ny, Nz//2+1)``
(src/hit3d/__init__.py:15-78), with torch CUDA tensors in place of JAX
arrays.  The package directory name starts with a digit, so import it with
``importlib.import_module("3dhit_b200")``.
"""

from ._native import DeviceWaitError, check_device
from .callbacks import Callback, Diagnostic, FieldWriter, State, save_series
from .diagnostics import (
    compensated_spectrum,
    component_spectra,
    dissipation,
    dissipation_constant,
    energy,
    energy_budget,
    energy_budget_cb,
    energy_spectrum,
    enstrophy,
    integral_lengthscale,
    kolmogorov_scale,
    longitudinal_autocorrelation,
    taylor_microscale,
    taylor_reynolds,
    taylor_reynolds_field,
    velocity_moments,
    velocity_samples,
)
from .fields import (
    cfl_dt,
    default_spectrum,
    hit_initial_field,
    random_field,
    rm_spectrum,
    spectral_state,
    taylor_green,
)
from .forcing import BandForcing, HoldEnergyForcing, LinearForcing, NoForcing
from .grid import (
    Grid,
    ddx,
    ddy,
    ddz,
    dealias,
    dealias_project,
    laplacian,
    make_grid,
    project,
    spectral_shape,
    to_physical,
    to_spectral,
)
from .integrators import SCHEMES, evolve, ifrk4_step, rk4_step, rollout
from .adjoint import rhs_vjp, rk4_step_vjp, rollout_autograd, rollout_vjp
from .navierstokes import NSParams, is_dealiased, linear_operator, make_ns_rhs

__all__ = [
    "Grid", "make_grid", "spectral_shape", "ddx", "ddy", "ddz", "laplacian",
    "dealias", "project", "dealias_project", "to_physical", "to_spectral",
    "spectral_state", "random_field", "taylor_green", "default_spectrum", "rm_spectrum",
    "hit_initial_field", "cfl_dt",
    "NoForcing", "LinearForcing", "BandForcing", "HoldEnergyForcing",
    "NSParams", "make_ns_rhs", "linear_operator", "is_dealiased",
    "rk4_step", "ifrk4_step", "SCHEMES", "rollout", "evolve", "rhs_vjp", "rk4_step_vjp", "rollout_vjp", "rollout_autograd",
    "State", "Callback", "Diagnostic", "FieldWriter", "save_series",
    "energy", "enstrophy", "dissipation", "energy_spectrum", "component_spectra",
    "compensated_spectrum", "dissipation_constant", "kolmogorov_scale",
    "taylor_microscale", "taylor_reynolds", "taylor_reynolds_field", "energy_budget",
    "energy_budget_cb", "velocity_samples", "velocity_moments",
    "longitudinal_autocorrelation", "integral_lengthscale", "check_device", "DeviceWaitError",
]
