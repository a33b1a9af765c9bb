"""Integrating-factor RK4 (the scheme src/hit3d/integrators.py:15-16 lists as
to do, on linear_operator, src/hit3d/navierstokes.py:100-103) on the CUDA
path against the oracle's restatement.

Tolerances (relative L2): float32 states 1e-5, float64 states 1e-12; the
Beltrami decay, which the scheme integrates exactly, 1e-12 in float64."""

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

FORCINGS = ("none", "linear", "band", "hold")


def _tol(npdt):
    return 1e-5 if npdt == np.float32 else 1e-12


def _forcings(h3, orc, name, nu):
    return {
        "none": (h3.NoForcing(), orc.NoForcing()),
        "linear": (h3.LinearForcing(A=0.1333), orc.LinearForcing(A=0.1333)),
        "band": (h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0), orc.BandForcing(0.1, 1.0, 2.0)),
        "hold": (h3.HoldEnergyForcing(E_target=1.5, nu=nu), orc.HoldEnergyForcing(1.5, nu)),
    }[name]


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("forcing", FORCINGS)
@pytest.mark.parametrize("dealiased", [True, False])
def test_ifrk4_step_matches_oracle(h3, orc, dtype, forcing, dealiased):
    npdt = np.float32 if dtype == torch.float32 else np.float64
    g = h3.make_grid(32, dtype=dtype)
    og = orc.make_grid(32, dtype=npdt)
    u0 = orc.hit_initial_field(0, og)
    nu, dt = 0.02, 4e-3
    f, of = _forcings(h3, orc, forcing, nu)
    u = h3.ifrk4_step(h3.make_ns_rhs(g), u0, h3.NSParams(nu=nu, forcing=f), dt, 0.0, assume_dealiased=dealiased)
    uo = orc.ifrk4_step(orc.make_ns_rhs(og), u0, orc.NSParams(nu=nu, forcing=of), dt, 0.0, og)
    assert rel_l2(_np(u), uo) < _tol(npdt)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_ifrk4_rollout_matches_oracle_and_differs_from_rk4(h3, orc, dtype):
    npdt = np.float32 if dtype == torch.float32 else np.float64
    g = h3.make_grid(32, dtype=dtype)
    og = orc.make_grid(32, dtype=npdt)
    u0 = orc.hit_initial_field(1, og)
    nu, dt, n = 0.05, 1e-2, 10
    f, of = _forcings(h3, orc, "band", nu)
    rhs, orhs = h3.make_ns_rhs(g), orc.make_ns_rhs(og)
    p, op = h3.NSParams(nu=nu, forcing=f), orc.NSParams(nu=nu, forcing=of)
    # the step graphs are rebuilt when the scheme changes
    u_rk = h3.rollout(rhs, u0, p, dt, n)
    u_if = h3.rollout(rhs, u0, p, dt, n, scheme="ifrk4")
    u_rk2 = h3.rollout(rhs, u0, p, dt, n)
    uo = u0
    for i in range(n):
        uo = orc.ifrk4_step(orhs, uo, op, dt, i * dt, og)
    assert rel_l2(_np(u_if), uo) < _tol(npdt)
    assert rel_l2(_np(u_rk), orc.rollout(orhs, u0, op, dt, n)) < _tol(npdt)
    assert torch.equal(u_rk, u_rk2)
    # both schemes are fourth order here (nu k_max^2 dt = 0.15): they differ at
    # the level of their truncation errors, visible above float64 rounding
    assert not torch.equal(u_if, u_rk)
    if npdt == np.float64:
        assert rel_l2(_np(u_if), _np(u_rk)) > 1e3 * _tol(npdt)


def test_ifrk4_beltrami_decay_is_exact_float64(h3, orc):
    # nu k_max^2 dt = 30 on the 32^3 box: far beyond RK4's stability limit
    g = h3.make_grid(32, dtype=torch.float64)
    u0 = torch.as_tensor(orc.beltrami(orc.make_grid(32, dtype=np.float64))).cuda()
    nu, dt, n = 0.5, 0.2, 20
    u = h3.rollout(h3.make_ns_rhs(g), u0, h3.NSParams(nu=nu), dt, n, scheme="ifrk4")
    assert rel_l2(_np(u), np.exp(-nu * dt * n) * _np(u0)) < 1e-12


def test_ifrk4_is_stable_where_rk4_is_not(h3, orc):
    g = h3.make_grid(16, dtype=torch.float64)
    og = orc.make_grid(16, dtype=np.float64)
    u0 = orc.hit_initial_field(2, og)
    kmax2 = float(np.max(og.k2 * og.dealias))
    nu = 0.2
    dt = 12.0 / (nu * kmax2)
    rhs = h3.make_ns_rhs(g)
    p = h3.NSParams(nu=nu)
    E0 = float(h3.energy(torch.as_tensor(u0).cuda(), g))
    u_if = h3.rollout(rhs, u0, p, dt, 10, scheme="ifrk4")
    u_rk = h3.rollout(rhs, u0, p, dt, 10)
    E_if, E_rk = float(h3.energy(u_if, g)), float(h3.energy(u_rk, g))
    assert np.isfinite(E_if) and E_if < E0
    assert not np.isfinite(E_rk) or E_rk > 1e3 * E0


def test_ifrk4_composed_path_matches_fused(h3, orc):
    class Custom:
        label = "custom"

        def term(self, u_hat, grid, t):
            return 0.1333 * u_hat

        def injection(self, u_hat, grid):
            return 0.0

    g = h3.make_grid(32)
    og = orc.make_grid(32, dtype=np.float32)
    u0 = torch.as_tensor(orc.hit_initial_field(3, og)).cuda()
    rhs = h3.make_ns_rhs(g)
    a = h3.ifrk4_step(rhs, u0, h3.NSParams(nu=0.02, forcing=Custom()), 4e-3, 0.0)
    b = h3.ifrk4_step(rhs, u0, h3.NSParams(nu=0.02, forcing=h3.LinearForcing(A=0.1333)), 4e-3, 0.0)
    assert rel_l2(_np(a), _np(b)) < 1e-5


def test_ifrk4_has_no_transpose(h3):
    nat = h3._native
    g = h3.make_grid(16)
    u = h3.spectral_state(g)
    p = h3.forcing.native_params(0.1, h3.NoForcing(), nat.HIT_FLAG_INTEGRATING_FACTOR)
    ub = torch.empty_like(u)
    with pytest.raises(Exception, match="no transpose"):
        nat.call("hit_rk4_step_vjp", g.plan.handle, nat.ptr(u), p, 1e-3, 0.0, nat.ptr(u), nat.ptr(ub), None,
                 nat.stream_ptr(g.device))
    with pytest.raises(ValueError):
        h3.rollout(h3.make_ns_rhs(g), u, h3.NSParams(nu=0.1), 1e-3, 1, scheme="etd")
