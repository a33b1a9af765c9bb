"""Host-side logic that needs no GPU: callback scheduling, evolve's segment
splitting (driven through a plain torch RHS on CPU tensors), forcing
parameter packing and its errors."""

import math
import importlib

import numpy as np
import pytest
import torch


def test_callback_schedules(h3):
    cb = h3.Callback(lambda s: None, every=3)
    assert [n for n in range(10) if cb.is_due(n, n * 0.1, 0.1)] == [0, 3, 6, 9]
    ct = h3.Callback(lambda s: None, every_time=0.25)
    due = [n for n in range(11) if ct.is_due(n, n * 0.1, 0.1)]
    assert due == [0, 3, 5, 8, 10]  # t crosses 0.25, 0.5, 0.75, 1.0
    with pytest.raises(ValueError):
        h3.Diagnostic(lambda s: 0.0, path="x.h5")


def test_evolve_segments_and_fires_callbacks(h3):
    # a linear decay RHS on CPU tensors goes through the generic RK4 path
    nu = 0.5
    rhs = lambda u, p, t: -p.nu * u  # noqa: E731
    p = h3.NSParams(nu=nu)
    u0 = torch.ones(4, dtype=torch.float64)
    seen = []
    d = h3.Diagnostic(lambda s: float(s.u_hat[0]), every=5)
    c = h3.Callback(lambda s: seen.append(s.step), every=4)
    u = h3.evolve(rhs, u0, p, None, 0.01, 12, callbacks=(d, c))
    assert seen == [0, 4, 8, 12]
    assert d.times == pytest.approx([0.0, 0.05, 0.10])
    # RK4 of du/dt = -nu u: per-step factor 1 - x + x^2/2 - x^3/6 + x^4/24
    x = nu * 0.01
    f = 1 - x + x**2 / 2 - x**3 / 6 + x**4 / 24
    assert float(u[0]) == pytest.approx(f**12, rel=1e-12)
    assert d.values[1] == pytest.approx(f**5, rel=1e-12)


def test_native_params_packing(h3):
    forcing = importlib.import_module("3dhit_b200.forcing")
    nat = importlib.import_module("3dhit_b200._native")
    p = forcing.native_params(0.01, h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0), nat.HIT_FLAG_ASSUME_DEALIASED)
    assert (p.forcing_kind, p.eps, p.kmin, p.kmax, p.flags) == (nat.HIT_FORCING_BAND, 0.1, 1.0, 2.0, 1)
    p = forcing.native_params(0.01, h3.HoldEnergyForcing(E_target=1.5, nu=0.01))
    assert p.forcing_kind == nat.HIT_FORCING_HOLD_ENERGY and p.E_target == 1.5 and p.tau == 0.0
    with pytest.raises(ValueError):
        forcing.native_params(0.02, h3.HoldEnergyForcing(E_target=1.5, nu=0.01))
    assert forcing.native_params(0.01, object()) is None  # custom forcing
    assert h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0).label == "BandForcing_eps0.1_k1-2"
    assert h3.NSParams(nu=1e-3).label == "NavierStokes_nu0.001_NoForcing"


def test_grid_arrays_match_oracle_on_cpu(h3, orc):
    for args, dt in (((32,), np.float32), ((16, 8, 4), np.float64)):
        g = h3.make_grid(*args, dtype=dt, device="cpu")
        og = orc.make_grid(*args, dtype=dt)
        for fld in ("kx", "ky", "kz", "k2", "inv_k2", "dealias", "weights"):
            np.testing.assert_array_equal(getattr(g, fld).numpy(), getattr(og, fld))
        assert g.num_shells == orc.shells(og)[1]
