"""CUDA path vs the reference's golden vectors and the float64 oracle.

Tolerances (relative L2 unless stated): float32 states 1e-5 (1 step and 100
steps), float64 states 1e-12; spectra and budgets of the same state 1e-6
against the reference's float32 values and 1e-11 against the float64
oracle.  Both code paths are exercised: the dealiased path (transforms skip
the modes outside the 2/3 box) and the general path (full transforms)."""

import numpy as np
import pytest
import torch

from conftest import CASES, rel_l2

pytestmark = pytest.mark.gpu

FORCINGS = ("none", "linear", "band")


def _state_tol(dt):
    return 1e-5 if np.dtype(dt) == np.float32 else 1e-12


def _forcing(h3, name):
    return {"none": h3.NoForcing(), "linear": h3.LinearForcing(A=0.1333),
            "band": h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0)}[name]


def _grid(h3, tag):
    dims, dt = CASES[tag]
    return h3.make_grid(*dims, dtype=torch.float32 if dt == np.float32 else torch.float64)


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("tag", list(CASES))
def test_transforms_match_reference(h3, golden, tag):
    g = _grid(h3, tag)
    tol = 1e-6 if CASES[tag][1] == np.float32 else 1e-13
    assert rel_l2(_np(h3.to_physical(golden[f"{tag}/u0"], g)), golden[f"{tag}/phys"]) < tol
    assert rel_l2(_np(h3.to_spectral(golden[f"{tag}/phys"], g)), golden[f"{tag}/spec_of_phys"]) < tol
    dp = _np(h3.dealias_project(golden[f"{tag}/spec_of_phys"], g))
    assert rel_l2(dp, golden[f"{tag}/dealias_project"]) < tol


@pytest.mark.parametrize("tag", list(CASES))
@pytest.mark.parametrize("forcing", FORCINGS)
@pytest.mark.parametrize("dealiased", [True, False])
def test_rhs_and_step_match_reference(h3, golden, tag, forcing, dealiased):
    g = _grid(h3, tag)
    nu, dt, _ = golden[f"{tag}/meta"]
    u0 = golden[f"{tag}/u0"]
    p = h3.NSParams(nu=float(nu), forcing=_forcing(h3, forcing))
    rhs = h3.make_ns_rhs(g)
    du = _np(rhs(u0, p, 0.0, assume_dealiased=dealiased))
    tol = _state_tol(CASES[tag][1])
    assert rel_l2(du, golden[f"{tag}/rhs_{forcing}"]) < tol
    u1 = _np(h3.rk4_step(rhs, u0, p, float(dt), 0.0, assume_dealiased=dealiased))
    assert rel_l2(u1, golden[f"{tag}/step_{forcing}"]) < tol
    # the dealias box stays exactly zero outside the mask
    mask = _np(g.dealias)
    assert np.all(u1[:, ~mask] == 0) or not dealiased


def test_auto_path_selection(h3, golden):
    g = _grid(h3, "c16f")
    u0 = torch.as_tensor(golden["c16f/u0"]).cuda()
    assert h3.is_dealiased(u0, g)
    v = u0.clone()
    v[0, 8, 0, 0] = 1e-3  # Nyquist x mode, outside the box
    assert not h3.is_dealiased(v, g)


def test_decay32_rollout_100_steps(h3, golden, orc):
    """Plain decaying HIT 32^3 (nu=0.02, dt=2e-3, 100 steps): state after 1,
    10 and 100 steps, spectra and budgets every 10 steps."""
    g = h3.make_grid(32)
    rhs = h3.make_ns_rhs(g)
    p = h3.NSParams(nu=0.02)
    u = torch.as_tensor(golden["decay32/u0"]).cuda()
    spectra, budgets = [], []
    for blk in range(10):
        _, E = h3.energy_spectrum(u, g)
        b = h3.energy_budget(u, g, 0.02, p.forcing)
        spectra.append(E)
        budgets.append([float(b["E"]), float(b["eps"]), float(b["P"])])
        u = h3.rollout(rhs, u, p, 2e-3, 10)
        if blk == 0:
            assert rel_l2(_np(u), golden["decay32/u10"]) < 1e-5
    _, E = h3.energy_spectrum(u, g)
    b = h3.energy_budget(u, g, 0.02, p.forcing)
    spectra.append(E)
    budgets.append([float(b["E"]), float(b["eps"]), float(b["P"])])
    err = rel_l2(_np(u), golden["decay32/u100"])
    assert err < 1e-5, err
    np.testing.assert_allclose(np.array(spectra), golden["decay32/spectra"], rtol=1e-5, atol=1e-12)
    np.testing.assert_allclose(np.array(budgets)[:, :2], golden["decay32/budgets"][:, :2], rtol=1e-5)
    # the same run in float64 by the oracle: error of the fp32 CUDA state vs fp64
    g64 = orc.make_grid(32, dtype=np.float64)
    u64 = orc.rollout(orc.make_ns_rhs(g64), golden["decay32/u0"].astype(np.complex128),
                      orc.NSParams(nu=0.02), 2e-3, 100)
    e64 = rel_l2(_np(u).astype(np.complex128), u64)
    print(f"decay32: rel-L2 vs reference fp32 {err:.3e}, vs fp64 oracle {e64:.3e}")
    assert e64 < 1e-5


@pytest.mark.parametrize("tag", list(CASES))
def test_diagnostics_match(h3, golden, orc, tag):
    g = _grid(h3, tag)
    dims, dt = CASES[tag]
    og = orc.make_grid(*dims, dtype=dt)
    u0 = golden[f"{tag}/u0"]
    nu = float(golden[f"{tag}/meta"][0])
    # vs the reference's own (float32/float64) values
    _, E = h3.energy_spectrum(u0, g)
    rt = 1e-6 if dt == np.float32 else 1e-12
    np.testing.assert_allclose(E, golden[f"{tag}/spectrum"], rtol=rt, atol=1e-14)
    _, e1, e2, e3 = h3.component_spectra(u0, g)
    np.testing.assert_allclose(np.stack([e1, e2, e3]), golden[f"{tag}/component_spectra"], rtol=rt, atol=1e-14)
    for name in FORCINGS:
        b = h3.energy_budget(u0, g, nu, _forcing(h3, name))
        np.testing.assert_allclose([float(b["E"]), float(b["eps"]), float(b["P"])],
                                   golden[f"{tag}/budget_{name}"], rtol=rt)
    # vs the float64 oracle on the same state
    _, E64, comp64 = orc.energy_spectrum_f64(u0, og)
    np.testing.assert_allclose(E, E64, rtol=1e-11, atol=1e-300)
    of = {"none": orc.NoForcing(), "linear": orc.LinearForcing(A=0.1333),
          "band": orc.BandForcing(eps=0.1, kmin=1.0, kmax=2.0),
          "hold": orc.HoldEnergyForcing(E_target=1.5, nu=nu)}
    hf = {"none": h3.NoForcing(), "linear": h3.LinearForcing(A=0.1333),
          "band": h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0),
          "hold": h3.HoldEnergyForcing(E_target=1.5, nu=nu)}
    for k in of:
        b = h3.energy_budget(u0, g, nu, hf[k])
        r = orc.energy_budget_f64(u0, og, nu, of[k])
        np.testing.assert_allclose([float(b["E"]), float(b["eps"]), float(b["P"])],
                                   [r["E"], r["eps"], r["P"]], rtol=1e-11)


def test_beltrami_float64(h3, orc):
    """reference tests/test_navierstokes.py:10-32 on the CUDA path (float64)."""
    g = h3.make_grid(32, dtype=torch.float64)
    u0 = torch.as_tensor(orc.beltrami(orc.make_grid(32, dtype=np.float64))).cuda()
    rhs = h3.make_ns_rhs(g)
    p = h3.NSParams(nu=0.05)
    du = rhs(u0, p, 0.0)
    assert torch.allclose(du, -0.05 * u0, atol=1e-10)
    u = h3.rollout(rhs, u0, p, 1e-2, 100)
    exact = np.exp(-0.05 * 1e-2 * 100) * _np(u0)
    assert rel_l2(_np(u), exact) < 1e-10


def test_invariants_and_inviscid_energy_float64(h3):
    """reference tests/test_navierstokes.py:35-54."""
    g = h3.make_grid(32, dtype=torch.float64)
    gen = torch.Generator(device="cuda").manual_seed(3)
    u = torch.randn((3, 32, 32, 32), generator=gen, dtype=torch.float64, device="cuda")
    u0 = h3.project(h3.dealias(h3.to_spectral(u, g), g), g)
    rhs = h3.make_ns_rhs(g)
    u = h3.rollout(rhs, u0, h3.NSParams(nu=0.02), 1e-3, 10)
    div = g.kx * u[0] + g.ky * u[1] + g.kz * u[2]
    assert float(div.abs().max()) < 1e-8
    assert torch.allclose(u * g.dealias, u)
    u = h3.rollout(rhs, u0, h3.NSParams(nu=0.0), 1e-3, 20)
    assert np.isclose(float(h3.energy(u, g)), float(h3.energy(u0, g)), rtol=1e-8)


def test_derivatives_roundtrip_anisotropic_float64(h3):
    """reference tests/test_grid.py:48-100."""
    g = h3.make_grid(32, dtype=torch.float64)
    N = 32
    x = (torch.arange(N, dtype=torch.float64, device="cuda") * (2 * np.pi / N)).reshape(-1, 1, 1)
    y = (torch.arange(N, dtype=torch.float64, device="cuda") * (2 * np.pi / N)).reshape(1, -1, 1)
    z = (torch.arange(N, dtype=torch.float64, device="cuda") * (2 * np.pi / N)).reshape(1, 1, -1)
    f = torch.sin(x) * torch.cos(2 * y) * torch.sin(3 * z)
    uh = h3.to_spectral(f.expand(3, N, N, N), g)
    assert torch.allclose(h3.to_physical(h3.ddx(uh, g), g)[0], torch.cos(x) * torch.cos(2 * y) * torch.sin(3 * z),
                          atol=1e-10)
    assert torch.allclose(h3.to_physical(h3.ddy(uh, g), g)[1], -2 * torch.sin(x) * torch.sin(2 * y) * torch.sin(3 * z),
                          atol=1e-10)
    assert torch.allclose(h3.to_physical(h3.ddz(uh, g), g)[2], 3 * torch.sin(x) * torch.cos(2 * y) * torch.cos(3 * z),
                          atol=1e-10)
    assert torch.allclose(h3.to_physical(h3.laplacian(uh, g), g)[0], -14 * f, atol=1e-9)
    ga = h3.make_grid(16, 8, 4, dtype=torch.float64)
    w = torch.randn((3, 16, 8, 4), dtype=torch.float64, device="cuda")
    assert torch.allclose(h3.to_physical(h3.to_spectral(w, ga), ga), w)


def test_projection_divergence_free_idempotent(h3):
    g = h3.make_grid(32, dtype=torch.float64)
    v = torch.randn((3, 32, 32, 17), dtype=torch.complex128, device="cuda")
    v = h3.project(v, g)
    assert float((g.kx * v[0] + g.ky * v[1] + g.kz * v[2]).abs().max()) < 1e-10
    assert torch.allclose(h3.project(v, g), v)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_device_random_field_spectrum(h3, dtype):
    """reference tests/test_diagnostics.py:31-43 on the device random_field."""
    g = h3.make_grid(32, dtype=dtype)
    u = h3.random_field(2, g)
    ks, Es = h3.energy_spectrum(u, g)
    rt = 1e-5 if dtype == torch.float32 else 1e-8
    np.testing.assert_allclose(Es[1:32 // 3], h3.default_spectrum(ks)[1:32 // 3], rtol=rt)
    assert np.isclose(Es.sum(), float(h3.energy(u, g)), rtol=rt)
    assert h3.is_dealiased(u, g)


def test_random_field_host_noise_matches_oracle(h3, orc):
    g = h3.make_grid(16, dtype=torch.float64)
    og = orc.make_grid(16, dtype=np.float64)
    u = _np(h3.random_field(5, g, host_noise=True))
    assert rel_l2(u, orc.random_field(5, og)) < 1e-12


def test_injection_exact(h3, orc):
    """reference tests/test_budget.py:39-60."""
    g = h3.make_grid(32, dtype=torch.float64)
    u = h3.random_field(0, g)
    f = h3.BandForcing(eps=0.3, kmin=1.0, kmax=3.0)
    assert float(f.injection(u, g)) == 0.3
    assert float(f.injection(torch.zeros_like(u), g)) == 0.0
    lf = h3.LinearForcing(A=0.1333)
    assert np.isclose(float(lf.injection(u, g)), 2 * 0.1333 * float(h3.energy(u, g)))
    # term/injection agree (plug-in API)
    n2 = float(32**3) ** 2

    def measured(term):
        return float((g.weights * (u.conj() * term).real.sum(0)).sum() / n2)

    assert np.isclose(measured(f.term(u, g, 0.0)), 0.3)
    hf = h3.HoldEnergyForcing(E_target=1.0, nu=0.05)
    assert np.isclose(measured(hf.term(u, g, 0.0)), float(hf.injection(u, g)))


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_hold_energy_forcing(h3, orc, dtype):
    """The hold-E Lundgren forcing keeps E at its target; matches the oracle."""
    g = h3.make_grid(32, dtype=dtype)
    npdt = np.float32 if dtype == torch.float32 else np.float64
    og = orc.make_grid(32, dtype=npdt)
    u0 = orc.hit_initial_field(0, og, k0=4.0)
    nu = 0.02
    p = h3.NSParams(nu=nu, forcing=h3.HoldEnergyForcing(E_target=1.5, nu=nu))
    u = h3.rollout(h3.make_ns_rhs(g), u0, p, 2e-3, 50)
    E = float(h3.energy(u, g))
    assert abs(E - 1.5) < (2e-5 if dtype == torch.float32 else 1e-10)
    uo = orc.rollout(orc.make_ns_rhs(og), u0, orc.NSParams(nu=nu, forcing=orc.HoldEnergyForcing(1.5, nu)),
                     2e-3, 50)
    assert rel_l2(_np(u), uo) < _state_tol(npdt)


def test_band_forced_rollout_matches_oracle(h3, orc):
    g = h3.make_grid(32)
    og = orc.make_grid(32, dtype=np.float32)
    u0 = orc.hit_initial_field(1, og)
    p = h3.NSParams(nu=6e-3, forcing=h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0))
    u = h3.rollout(h3.make_ns_rhs(g), u0, p, 2e-3, 20)
    uo = orc.rollout(orc.make_ns_rhs(og), u0, orc.NSParams(nu=6e-3, forcing=orc.BandForcing(0.1, 1.0, 2.0)),
                     2e-3, 20)
    assert rel_l2(_np(u), uo) < 1e-5


def test_custom_forcing_goes_through_projection(h3, golden):
    class Custom:
        label = "custom"

        def term(self, u_hat, grid, t):
            return 0.1333 * u_hat

        def injection(self, u_hat, grid):
            return 0.0

    g = _grid(h3, "c16f")
    u0 = golden["c16f/u0"]
    nu = float(golden["c16f/meta"][0])
    rhs = h3.make_ns_rhs(g)
    a = rhs(u0, h3.NSParams(nu=nu, forcing=Custom()), 0.0)
    b = rhs(u0, h3.NSParams(nu=nu, forcing=h3.LinearForcing(A=0.1333)), 0.0)
    assert rel_l2(_np(a), _np(b)) < 1e-6
    # a custom rhs callable integrates through the generic stage algebra
    u1 = h3.rk4_step(lambda u, p, t: rhs(u, p, t), u0, h3.NSParams(nu=nu), 2e-3, 0.0)
    assert rel_l2(_np(u1), golden["c16f/step_none"]) < 1e-5


def test_errors_are_loud(h3):
    with pytest.raises(Exception, match="powers of two"):
        h3.make_grid(12).plan
    g = h3.make_grid(16)
    with pytest.raises(ValueError):
        h3.make_ns_rhs(g)(torch.zeros((3, 16, 16, 8), dtype=torch.complex64, device="cuda"),
                          h3.NSParams(nu=0.1), 0.0)
    with pytest.raises(ValueError):
        h3.rk4_step(h3.make_ns_rhs(g), h3.spectral_state(g),
                    h3.NSParams(nu=0.1, forcing=h3.HoldEnergyForcing(1.0, nu=0.2)), 1e-3, 0.0)
