"""Parity at the benchmark sizes: one RK4 step of the 512^3 band-forced
workload and of the 256^3 hold-energy workload on the CUDA path against the
float32 CPU oracle on the same initial field (the oracle takes a few tens of
seconds per step on the host cores at 512^3).

Tolerances: state relative L2 1e-5 (the float32 bar of the small-grid parity
tests); spectra and budgets of the same state (CUDA float64 sums against the
oracle's float64 sums) 1e-10 relative; spectra of the two stepped states
1e-6 of the total energy per shell; E, eps and P of the two stepped states
1e-6 relative."""

import gc

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def _step_case(h3, orc, N, nu, forcing_dev, forcing_orc, seed):
    g = h3.make_grid(N)
    u0 = h3.hit_initial_field(seed, g)
    dt = h3.cfl_dt(u0, g, 0.5)
    p = h3.NSParams(nu=nu, forcing=forcing_dev)
    u1 = h3.rk4_step(h3.make_ns_rhs(g), u0, p, dt, 0.0)
    _, E_dev = h3.energy_spectrum(u1, g)
    b_dev = {k: float(v) for k, v in h3.energy_budget(u1, g, nu, forcing_dev).items()}
    u0_h, u1_h = _np(u0), _np(u1)
    del u0, u1
    gc.collect()
    torch.cuda.empty_cache()

    og = orc.make_grid(N, dtype=np.float32)
    uo = orc.rk4_step(orc.make_ns_rhs(og), u0_h, orc.NSParams(nu=nu, forcing=forcing_orc), float(dt), 0.0)
    err = rel_l2(u1_h, uo)
    # the same state through both reductions
    _, E_same, _ = orc.energy_spectrum_f64(u1_h, og)
    same = float(np.max(np.abs(E_dev - E_same)) / E_same.sum())
    # the two stepped states
    _, E_orc, _ = orc.energy_spectrum_f64(uo, og)
    spec = float(np.max(np.abs(E_dev - E_orc)) / E_orc.sum())
    b_orc = orc.energy_budget_f64(uo, og, nu, forcing_orc)
    bud = {k: abs(b_dev[k] - float(b_orc[k])) / abs(float(b_orc[k])) for k in ("E", "eps", "P")}
    print(f"{N}^3 one RK4 step (dt {dt:.3e}): state rel-L2 {err:.2e}; spectrum of the same state {same:.2e}; "
          f"spectra of the stepped states {spec:.2e} of E; budget {bud}")
    return err, same, spec, bud


def test_band_forced_512_one_step_vs_oracle(h3, orc):
    """The benchmark workload itself (512^3, BandForcing eps=0.1 k in [1, 2],
    nu = 6e-4, dt from CFL 0.5) against the oracle."""
    f = dict(eps=0.1, kmin=1.0, kmax=2.0)
    err, same, spec, bud = _step_case(h3, orc, 512, 6e-4, h3.BandForcing(**f), orc.BandForcing(**f), 0)
    assert err < 1e-5
    assert same < 1e-10
    assert spec < 1e-6
    assert max(bud.values()) < 1e-6, bud


def test_hold_energy_256_one_step_vs_oracle(h3, orc):
    """The Lundgren hold-energy workload (256^3, E_t = 1.5, nu = 1.5e-3, dt
    from CFL 0.5) against the oracle (float64 coefficient on both sides)."""
    nu = 1.5e-3
    err, same, spec, bud = _step_case(h3, orc, 256, nu, h3.HoldEnergyForcing(E_target=1.5, nu=nu),
                                      orc.HoldEnergyForcing(E_target=1.5, nu=nu), 1)
    assert err < 1e-5
    assert same < 1e-10
    assert spec < 1e-6
    assert max(bud.values()) < 1e-6, bud
