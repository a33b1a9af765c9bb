"""Oracle checks of the integrating-factor RK4 scheme (no reference
implementation: src/hit3d/integrators.py:15-16 lists it as to do, on top of
linear_operator, src/hit3d/navierstokes.py:100-103).  CPU only."""

import numpy as np
import pytest

from conftest import rel_l2


@pytest.fixture(scope="module")
def g16(orc):
    return orc.make_grid(16, dtype=np.float64)


def _random_state(orc, g, seed):
    rng = np.random.default_rng(seed)
    N = g.Nx
    u = orc.to_spectral(rng.standard_normal((3, N, N, N)), g)
    return orc.project(orc.dealias(u, g), g)


def test_ifrk4_at_zero_viscosity_is_rk4(orc, g16):
    # E = 1: every stage input and the combination reduce to the RK4 ones
    u0 = _random_state(orc, g16, 0)
    rhs = orc.make_ns_rhs(g16)
    p = orc.NSParams(nu=0.0)
    a = orc.ifrk4_step(rhs, u0, p, 1e-3, 0.0, g16)
    b = orc.rk4_step(rhs, u0, p, 1e-3, 0.0)
    np.testing.assert_array_equal(a, b)


def test_ifrk4_beltrami_decay_is_exact(orc):
    # u x w = 0 for a Beltrami field: the step is exp(-nu k^2 dt) u exactly,
    # even at nu k_max^2 dt = 30, where RK4 is unstable
    g = orc.make_grid(32, dtype=np.float64)
    u0 = orc.beltrami(g)
    rhs = orc.make_ns_rhs(g)
    nu, dt, n = 0.5, 0.2, 20
    p = orc.NSParams(nu=nu)
    u = u0
    for i in range(n):
        u = orc.ifrk4_step(rhs, u, p, dt, i * dt, g)
    exact = np.exp(-nu * dt * n) * u0
    assert rel_l2(u, exact) < 1e-12


def test_ifrk4_is_stable_beyond_the_rk4_viscous_limit(orc, g16):
    # nu k_max^2 dt = 12 > 2.785 (RK4's real-axis limit): RK4 grows, IF-RK4 decays
    u0 = _random_state(orc, g16, 1)
    rhs = orc.make_ns_rhs(g16)
    kmax2 = float(np.max(g16.k2 * g16.dealias))
    nu = 0.2
    dt = 12.0 / (nu * kmax2)
    p = orc.NSParams(nu=nu)
    E0 = orc.energy(u0, g16)
    u_if, u_rk = u0, u0
    with np.errstate(over="ignore", invalid="ignore"):
        for i in range(10):
            u_if = orc.ifrk4_step(rhs, u_if, p, dt, i * dt, g16)
            u_rk = orc.rk4_step(rhs, u_rk, p, dt, i * dt)
        E_rk = orc.energy(u_rk, g16)
    assert np.isfinite(u_if).all() and orc.energy(u_if, g16) < E0
    assert not np.isfinite(E_rk) or E_rk > 1e3 * E0


def test_ifrk4_is_fourth_order(orc, g16):
    u0 = _random_state(orc, g16, 2) * 0.3
    rhs = orc.make_ns_rhs(g16)
    p = orc.NSParams(nu=0.05, forcing=orc.LinearForcing(A=0.1))
    T = 0.2

    def run(n):
        dt = T / n
        u = u0
        for i in range(n):
            u = orc.ifrk4_step(rhs, u, p, dt, i * dt, g16)
        return u

    ref = run(64)
    e1, e2 = rel_l2(run(4), ref), rel_l2(run(8), ref)
    assert 11.0 < e1 / e2 < 22.0, (e1, e2)


def test_ifrk4_float32_follows_float64(orc):
    g32 = orc.make_grid(16, dtype=np.float32)
    g64 = orc.make_grid(16, dtype=np.float64)
    u64 = _random_state(orc, g64, 3)
    u32 = u64.astype(np.complex64)
    f = orc.BandForcing(eps=0.1, kmin=1.0, kmax=2.0)
    p = orc.NSParams(nu=0.02, forcing=f)
    a = orc.ifrk4_step(orc.make_ns_rhs(g32), u32, p, 5e-3, 0.0, g32)
    b = orc.ifrk4_step(orc.make_ns_rhs(g64), u64, p, 5e-3, 0.0, g64)
    assert a.dtype == np.complex64
    assert rel_l2(a, b) < 1e-5
