"""The benchmark configurations at their own sizes, through size-independent
properties (the CPU oracle cannot run them in test time), plus the evolve /
callback path and float32-vs-float64 error statements."""

import math

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def test_evolve_budget_residual_float64(h3, orc):
    """reference tests/test_budget.py:82-95 through evolve + Diagnostic."""
    g = h3.make_grid(32, dtype=torch.float64)
    u = torch.as_tensor(orc.random_field(2, orc.make_grid(32, dtype=np.float64))).cuda()
    d = h3.Diagnostic(h3.energy_budget_cb, every=1)
    dt, nsteps = 1e-3, 50
    h3.evolve(h3.make_ns_rhs(g), u, h3.NSParams(nu=0.05), g, dt, nsteps, callbacks=(d,))
    E = np.array([v["E"] for v in d.values])
    eps = np.array([v["eps"] for v in d.values])
    assert len(E) == nsteps + 1
    resid = (E[2:] - E[:-2]) / (2 * dt) + eps[1:-1]
    assert np.max(np.abs(resid)) < 1e-4 * eps.max()


def test_band_forced_512_properties(h3):
    """Band-forced HIT at 512^3 (the benchmark case): the dealiased and the
    general code paths agree, the state stays in the 2/3 box and divergence
    free, and the energy changes by dt (P - eps) to RK4 accuracy."""
    g = h3.make_grid(512)
    u0 = h3.hit_initial_field(0, g)
    dt = h3.cfl_dt(u0, g, 0.5)
    p = h3.NSParams(nu=6e-4, forcing=h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0))
    rhs = h3.make_ns_rhs(g)
    b0 = h3.energy_budget(u0, g, p.nu, p.forcing)
    u1 = h3.rollout(rhs, u0, p, dt, 2, assume_dealiased=True)
    u1g = h3.rollout(rhs, u0, p, dt, 2, assume_dealiased=False)
    err = float(torch.linalg.vector_norm(u1 - u1g) / torch.linalg.vector_norm(u1g))
    assert err < 1e-5, err
    del u1g
    torch.cuda.empty_cache()
    assert h3.is_dealiased(u1, g)
    kx = g.kx.to(torch.complex64)
    div = (kx * u1[0] + g.ky * u1[1] + g.kz * u1[2]).abs().max()
    kmag = torch.sqrt(g.k2).max()
    assert float(div) < 1e-6 * float(kmag * u1.abs().max())
    b1 = h3.energy_budget(u1, g, p.nu, p.forcing)
    assert float(b0["P"]) == pytest.approx(0.1)
    dE = float(b1["E"]) - float(b0["E"])
    expect = 2 * dt * 0.5 * (float(b0["P"] - b0["eps"]) + float(b1["P"] - b1["eps"]))
    assert dE == pytest.approx(expect, rel=2e-2, abs=1e-7)
    _, E = h3.energy_spectrum(u1, g)
    assert E.sum() == pytest.approx(float(b1["E"]), rel=1e-10)


def test_hold_energy_256(h3):
    """Lundgren hold-E forcing at 256^3 (the configuration's forcing and size):
    E stays at its target through a CUDA-graph rollout."""
    g = h3.make_grid(256)
    u0 = h3.hit_initial_field(0, g)
    nu = 1.5e-3
    p = h3.NSParams(nu=nu, forcing=h3.HoldEnergyForcing(E_target=1.5, nu=nu))
    dt = h3.cfl_dt(u0, g, 0.5)
    u = h3.rollout(h3.make_ns_rhs(g), u0, p, dt, 20)
    b = h3.energy_budget(u, g, nu, p.forcing)
    assert float(b["E"]) == pytest.approx(1.5, rel=2e-6)
    assert float(b["P"]) == pytest.approx(float(b["eps"]), rel=1e-9)  # tau = inf: P = eps


def test_fp32_error_against_fp64_same_solver(h3, orc):
    """Error of the float32 CUDA state against a float64 run of the same
    solver (and that float64 run against the float64 oracle)."""
    N, nsteps = 64, 20
    og = orc.make_grid(N, dtype=np.float64)
    u0 = orc.hit_initial_field(3, og)
    p = dict(nu=6e-3)
    g32, g64 = h3.make_grid(N), h3.make_grid(N, dtype=torch.float64)
    f = dict(eps=0.1, kmin=1.0, kmax=2.0)
    u32 = h3.rollout(h3.make_ns_rhs(g32), u0.astype(np.complex64), h3.NSParams(forcing=h3.BandForcing(**f), **p),
                     2e-3, nsteps)
    u64 = h3.rollout(h3.make_ns_rhs(g64), u0, h3.NSParams(forcing=h3.BandForcing(**f), **p), 2e-3, nsteps)
    uo = orc.rollout(orc.make_ns_rhs(og), u0, orc.NSParams(nu=6e-3, forcing=orc.BandForcing(**f)), 2e-3, nsteps)
    e32 = rel_l2(_np(u32).astype(np.complex128), _np(u64))
    e64 = rel_l2(_np(u64), uo)
    _, E32 = h3.energy_spectrum(u32, g32)
    _, E64 = h3.energy_spectrum(u64, g64)
    espec = float(np.max(np.abs(E32 - E64)) / E64.sum())           # relative to the total energy
    eres = float(np.max(np.abs(E32 - E64)[: N // 3] / E64[: N // 3]))  # per shell, resolved shells
    print(f"64^3 band, {nsteps} steps: fp32 vs fp64 state {e32:.2e}, spectrum {espec:.2e} of E "
          f"(per resolved shell {eres:.2e}); fp64 CUDA vs fp64 oracle {e64:.2e}")
    assert e32 < 1e-5 and e64 < 1e-11
    assert espec < 1e-6 and eres < 1e-5
