"""evolve + callbacks on the GPU (the reference's tests/test_callbacks.py
scenarios on a Beltrami field, with the in-memory ``h5py`` stand-in), and the
physical-space diagnostics against the reference's own outputs
(``tests/golden/reference_aux.npz``: velocity_samples, velocity_moments,
longitudinal_autocorrelation, integral_lengthscale of
src/hit3d/diagnostics.py:188-244)."""

import os
import sys

import numpy as np
import pytest
import torch

from conftest import REPO, rel_l2

pytestmark = pytest.mark.gpu

NU = 0.05


@pytest.fixture
def h5(monkeypatch):
    import h5stub
    monkeypatch.setitem(sys.modules, "h5py", h5stub)
    return h5stub


def _beltrami(h3, orc, N=32):
    g = h3.make_grid(N, dtype=torch.float64)
    return g, torch.as_tensor(orc.beltrami(orc.make_grid(N, dtype=np.float64))).cuda()


def test_scheduling_snapshots_and_series(h3, orc, h5, tmp_path):
    g, u0 = _beltrami(h3, orc)
    dt, nsteps = 1e-2, 100
    E = h3.Diagnostic(lambda s: h3.energy(s.u_hat, s.grid), every=10)
    steps = []
    probe = h3.Callback(lambda s: steps.append(s.step), every_time=0.25)
    path = str(tmp_path / "snap.h5")
    writer = h3.FieldWriter(path, every=50)
    budget = h3.Diagnostic(h3.energy_budget_cb, every=25, path=path, name="budget")
    u = h3.evolve(h3.make_ns_rhs(g), u0, h3.NSParams(nu=NU), g, dt, nsteps, callbacks=(E, probe, writer, budget))
    # energy decays as e^{-2 nu t} (Beltrami: u x w = 0)
    assert len(E.times) == nsteps // 10 + 1 and E.times[1] == pytest.approx(10 * dt)
    expect = E.values[0] * np.exp(-2 * NU * np.asarray(E.times))
    np.testing.assert_allclose(np.asarray(E.values), expect, rtol=1e-8)
    assert steps == [0, 25, 50, 75, 100]
    with h5.File(path, "r") as f:
        assert sorted(k for k in f if k.startswith("step_")) == ["step_00000000", "step_00000050",
                                                                    "step_00000100"]
        np.testing.assert_array_equal(f["step_00000100/u_hat"][()], u.cpu().numpy())
        assert f["step_00000100/t"][()] == pytest.approx(dt * nsteps)
        assert f["grid/Nx"][()] == 32 and f["grid/nu"][()] == NU
        np.testing.assert_allclose(f["series/budget/t"][()], [0.0, 0.25, 0.5, 0.75, 1.0])
        np.testing.assert_allclose(f["series/budget/E"][()], [v["E"] for v in budget.values])


def test_time_scheduled_snapshots(h3, orc, h5, tmp_path):
    g, u0 = _beltrami(h3, orc)
    path = str(tmp_path / "snap.h5")
    h3.evolve(h3.make_ns_rhs(g), u0, h3.NSParams(nu=NU), g, 0.1, 30,
              callbacks=(h3.FieldWriter(path, every_time=0.5, warmup_time=1.0),))
    with h5.File(path, "r") as f:
        steps = sorted(k for k in f if k.startswith("step_"))
    assert steps == [f"step_{s:08d}" for s in (10, 15, 20, 25, 30)]


def test_deferred_diagnostics_equal_direct_reads(h3):
    """Diagnostic values fetched in one batch at the end equal per-step reads."""
    g = h3.make_grid(32)
    u0 = h3.hit_initial_field(0, g)
    p = h3.NSParams(nu=0.02, forcing=h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0))
    rhs = h3.make_ns_rhs(g)
    spec = h3.Diagnostic(lambda s: h3.energy_spectrum(s.u_hat, s.grid)[1], every=5)
    dev = h3.Diagnostic(lambda s: torch.stack(list(h3.energy_budget(s.u_hat, s.grid, 0.02, p.forcing).values())),
                        every=5)
    u = h3.evolve(rhs, u0, p, g, 2e-3, 20, callbacks=(spec, dev))
    assert len(spec.values) == len(dev.values) == 5
    b = h3.energy_budget(u, g, 0.02, p.forcing)
    np.testing.assert_allclose(dev.values[-1], [float(b["E"]), float(b["eps"]), float(b["P"])], rtol=0, atol=0)
    np.testing.assert_allclose(spec.values[-1], h3.energy_spectrum(u, g)[1], rtol=0, atol=0)


AUX = os.path.join(REPO, "tests", "golden", "reference_aux.npz")


@pytest.mark.parametrize("tag", ["c16f", "a16x32x8f", "c16d"])
def test_physical_space_diagnostics_match_reference(h3, tag):
    aux = np.load(AUX)
    u0 = aux[f"{tag}/u0"]
    f64 = u0.dtype == np.complex128
    g = h3.make_grid(*[2 * (s - 1) if i == 2 else s for i, s in enumerate(u0.shape[1:])],
                     dtype=torch.float64 if f64 else torch.float32)
    tol = 1e-12 if f64 else 2e-6
    for c in range(3):
        smp = h3.velocity_samples(u0, g, component=c)
        assert rel_l2(smp, aux[f"{tag}/samples{c}"]) < tol
        mom = h3.velocity_moments(smp)
        ref = aux[f"{tag}/moments{c}"]
        got = np.array([mom[k] for k in ("mean", "variance", "skewness", "flatness")], dtype=np.float64)
        # the mean of a zero-mean field is roundoff: compare it on the scale of the rms
        assert abs(got[0] - ref[0]) < 1e3 * tol * np.sqrt(ref[1])
        np.testing.assert_allclose(got[1:], ref[1:], rtol=50 * tol)
        r, f = h3.longitudinal_autocorrelation(u0, g, component=c)
        np.testing.assert_allclose(r, aux[f"{tag}/autocorr_r{c}"], rtol=1e-15)
        np.testing.assert_allclose(f, aux[f"{tag}/autocorr_f{c}"], rtol=0, atol=10 * tol)
        L = h3.integral_lengthscale(r, f)
        assert L == pytest.approx(float(aux[f"{tag}/lengthscale{c}"][0]), rel=100 * tol, abs=1e-12)
