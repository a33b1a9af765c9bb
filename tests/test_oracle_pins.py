"""The CPU oracle against (1) golden vectors made by the reference's own code
(tests/golden/make_golden.py) and (2) the reference's analytic known-answer
tests (tests/test_grid.py, test_navierstokes.py, test_diagnostics.py,
test_budget.py of the reference), ported onto the oracle in float64."""

import numpy as np
import pytest

from conftest import CASES, rel_l2


def _tol(dt):
    return 1e-6 if np.dtype(dt) == np.float32 else 1e-13


@pytest.mark.parametrize("tag", list(CASES))
def test_oracle_matches_reference_vectors(tag, orc, golden):
    dims, dt = CASES[tag]
    g = orc.make_grid(*dims, dtype=dt)
    u0 = golden[f"{tag}/u0"]
    nu, dtt, _ = golden[f"{tag}/meta"]
    assert rel_l2(orc.to_physical(u0, g), golden[f"{tag}/phys"]) < _tol(dt)
    rhs = orc.make_ns_rhs(g)
    forcings = {"none": orc.NoForcing(), "linear": orc.LinearForcing(A=0.1333),
                "band": orc.BandForcing(eps=0.1, kmin=1.0, kmax=2.0)}
    for name, f in forcings.items():
        p = orc.NSParams(nu=nu, forcing=f)
        assert rel_l2(rhs(u0, p, 0.0), golden[f"{tag}/rhs_{name}"]) < _tol(dt)
        assert rel_l2(orc.rk4_step(rhs, u0, p, dtt, 0.0), golden[f"{tag}/step_{name}"]) < _tol(dt)
        b = orc.energy_budget(u0, g, nu, f)
        np.testing.assert_allclose([float(b["E"]), float(b["eps"]), float(b["P"])],
                                   golden[f"{tag}/budget_{name}"], rtol=10 * _tol(dt), atol=1e-30)
    np.testing.assert_allclose(orc.energy_spectrum(u0, g)[1], golden[f"{tag}/spectrum"], rtol=_tol(dt), atol=1e-30)


def test_oracle_grid_arrays_match_reference(orc, golden):
    for tag, args, dt in (("g32f", (32,), np.float32), ("g16x8x4d", (16, 8, 4), np.float64),
                          ("g8f", (8,), np.float32)):
        g = orc.make_grid(*args, dtype=dt)
        for fld in ("kx", "ky", "kz", "k2", "inv_k2", "dealias", "weights"):
            np.testing.assert_array_equal(getattr(g, fld), golden[f"{tag}/{fld}"])


def test_oracle_decay32_rollout(orc, golden):
    """100 steps of the plain decaying 32^3 config match the reference run."""
    g = orc.make_grid(32, dtype=np.float32)
    rhs = orc.make_ns_rhs(g)
    p = orc.NSParams(nu=0.02)
    u = orc.rollout(rhs, golden["decay32/u0"], p, 2e-3, 10)
    assert rel_l2(u, golden["decay32/u10"]) < 1e-6
    u = orc.rollout(rhs, u, p, 2e-3, 90, 10 * 2e-3)
    assert rel_l2(u, golden["decay32/u100"]) < 1e-5


# --- the reference's analytic tests, on the oracle (float64, 32^3) ---------

N = 32
NU = 0.05


@pytest.fixture(scope="module")
def g64(orc):
    return orc.make_grid(32, dtype=np.float64)


def test_beltrami_rhs_is_pure_viscous_decay(orc, g64):
    # reference tests/test_navierstokes.py:10-19
    u0 = orc.beltrami(g64)
    du = orc.make_ns_rhs(g64)(u0, orc.NSParams(nu=NU), 0.0)
    np.testing.assert_allclose(du, -NU * u0, atol=1e-10)


def test_beltrami_decay_matches_analytic(orc, g64):
    # reference tests/test_navierstokes.py:22-32
    u0 = orc.beltrami(g64)
    dt, n = 1e-2, 100
    u = orc.rollout(orc.make_ns_rhs(g64), u0, orc.NSParams(nu=NU), dt, n)
    assert rel_l2(u, np.exp(-NU * dt * n) * u0) < 1e-10


def test_rollout_invariants_and_inviscid_energy(orc, g64):
    # reference tests/test_navierstokes.py:35-54
    rng = np.random.default_rng(3)
    u0 = orc.project(orc.dealias(orc.to_spectral(rng.standard_normal((3, N, N, N)), g64), g64), g64)
    rhs = orc.make_ns_rhs(g64)
    u = orc.rollout(rhs, u0, orc.NSParams(nu=0.02), 1e-3, 10)
    div = g64.kx * u[0] + g64.ky * u[1] + g64.kz * u[2]
    assert np.max(np.abs(div)) < 1e-8
    np.testing.assert_allclose(u * g64.dealias, u)
    u = orc.rollout(rhs, u0, orc.NSParams(nu=0.0), 1e-3, 20)
    assert np.isclose(orc.energy(u, g64), orc.energy(u0, g64), rtol=1e-8)


def test_transforms_and_operators(orc, g64):
    # reference tests/test_grid.py:48-100
    rng = np.random.default_rng(0)
    u = rng.standard_normal((3, N, N, N))
    np.testing.assert_allclose(orc.to_physical(orc.to_spectral(u, g64), g64), u, atol=1e-12)
    x = (np.arange(N) * (2 * np.pi / N)).reshape(-1, 1, 1)
    y = (np.arange(N) * (2 * np.pi / N)).reshape(1, -1, 1)
    z = (np.arange(N) * (2 * np.pi / N)).reshape(1, 1, -1)
    f = np.sin(x) * np.cos(2 * y) * np.sin(3 * z)
    uh = orc.to_spectral(np.broadcast_to(f, (3, N, N, N)), g64)
    np.testing.assert_allclose(orc.to_physical(orc.ddx(uh, g64), g64)[0],
                               np.cos(x) * np.cos(2 * y) * np.sin(3 * z), atol=1e-10)
    np.testing.assert_allclose(orc.to_physical(orc.laplacian(uh, g64), g64)[0], -14 * f, atol=1e-9)
    v = rng.standard_normal((3, N, N, N // 2 + 1)) + 1j * rng.standard_normal((3, N, N, N // 2 + 1))
    v = orc.project(v, g64)
    assert np.max(np.abs(g64.kx * v[0] + g64.ky * v[1] + g64.kz * v[2])) < 1e-10
    assert np.allclose(orc.project(v, g64), v)
    ga = orc.make_grid(16, 8, 4, dtype=np.float64)
    w = rng.standard_normal((3, 16, 8, 4))
    np.testing.assert_allclose(orc.to_physical(orc.to_spectral(w, ga), ga), w, atol=1e-12)


def test_parseval_spectrum_ic(orc, g64):
    # reference tests/test_diagnostics.py:23-43
    rng = np.random.default_rng(0)
    u = rng.standard_normal((3, N, N, N))
    assert np.isclose(orc.energy(orc.to_spectral(u, g64), g64), 0.5 * np.sum(u**2) / N**3)
    uh = orc.random_field(1, g64)
    assert np.isclose(orc.energy_spectrum(uh, g64)[1].sum(), orc.energy(uh, g64))
    uh = orc.random_field(2, g64)
    ks, Es = orc.energy_spectrum(uh, g64)
    np.testing.assert_allclose(Es[1:N // 3], orc.default_spectrum(ks)[1:N // 3], rtol=1e-8)


def test_injection_exact_and_budget_residual(orc, g64):
    # reference tests/test_budget.py:39-95
    uh = orc.random_field(0, g64)
    n2 = float(N**3) ** 2

    def measured(term):
        return float(np.sum(g64.weights * np.sum(np.real(np.conj(uh) * term), axis=0)) / n2)

    f = orc.BandForcing(eps=0.3, kmin=1.0, kmax=3.0)
    assert float(f.injection(uh, g64)) == 0.3
    assert float(f.injection(np.zeros_like(uh), g64)) == 0.0
    assert np.isclose(measured(f.term(uh, g64, 0.0)), 0.3)
    lf = orc.LinearForcing(A=0.1333)
    assert np.isclose(lf.injection(uh, g64), 2 * 0.1333 * orc.energy(uh, g64))
    hf = orc.HoldEnergyForcing(E_target=1.0, nu=NU)
    assert np.isclose(measured(hf.term(uh, g64, 0.0)), float(hf.injection(uh, g64)))
    # finite-difference budget residual over a short decay
    rhs = orc.make_ns_rhs(g64)
    p = orc.NSParams(nu=NU)
    E, eps = [], []
    u = orc.random_field(2, g64)
    for _ in range(51):
        b = orc.energy_budget(u, g64, NU, p.forcing)
        E.append(float(b["E"])); eps.append(float(b["eps"]))
        u = orc.rk4_step(rhs, u, p, 1e-3, 0.0)
    E, eps = np.array(E), np.array(eps)
    resid = (E[2:] - E[:-2]) / 2e-3 + eps[1:-1]
    assert np.max(np.abs(resid)) < 1e-4 * eps.max()


def test_hold_energy_holds_energy(orc):
    g = orc.make_grid(16, dtype=np.float64)
    u = orc.hit_initial_field(0, g, k0=2.0)
    nu = 0.02
    p = orc.NSParams(nu=nu, forcing=orc.HoldEnergyForcing(E_target=1.5, nu=nu))
    u2 = orc.rollout(orc.make_ns_rhs(g), u, p, 2e-3, 20)
    assert abs(orc._energy_enstrophy_f64(u2, g)[0] - 1.5) < 1e-8
