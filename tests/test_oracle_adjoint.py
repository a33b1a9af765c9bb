"""The oracle's discrete adjoint against central finite differences (CPU).

The reference differentiates its RHS, RK4 step and rollout with jax.vjp
(src/hit3d/navierstokes.py:62-97, src/hit3d/integrators.py:32-53); jax is not
installable here, so the oracle's hand-written transpose is pinned by finite
differences of the oracle's own forward functions, in float64, along random
directions that are neither Hermitian nor dealiased.  Cotangents are
dL/dRe + i dL/dIm of the stored entries (inner product sum Re(conj(a) b)).
"""
import dataclasses

import numpy as np
import pytest


def _rc(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


FORCINGS = ["none", "linear", "band", "hold"]


def _params(orc, kind, nu=0.02, A=0.3, eps=0.1, tau=0.7):
    f = {"none": orc.NoForcing(), "linear": orc.LinearForcing(A), "band": orc.BandForcing(eps, 1.0, 2.0),
         "hold": orc.HoldEnergyForcing(1.5, nu, tau=tau)}[kind]
    return orc.NSParams(nu=nu, forcing=f)


@pytest.fixture(scope="module")
def case(orc):
    g = orc.make_grid(12, 10, 8, dtype=np.float64)
    rng = np.random.default_rng(7)
    u = orc.random_field(3, g)
    return g, u, rng


@pytest.mark.parametrize("kind", FORCINGS)
def test_rhs_vjp_state(orc, case, kind):
    g, u, rng = case
    p = _params(orc, kind)
    rhs = orc.make_ns_rhs(g)
    v, d = _rc(rng, u.shape), _rc(rng, u.shape)
    ub, _ = orc.rhs_vjp(g, u, p, v)
    h = 1e-6
    fd = (orc._dot_re(v, rhs(u + h * d, p, 0.0)) - orc._dot_re(v, rhs(u - h * d, p, 0.0))) / (2 * h)
    assert abs(orc._dot_re(ub, d) - fd) <= 1e-7 * abs(fd)


@pytest.mark.parametrize("kind,name", [("none", "nu"), ("linear", "A"), ("linear", "nu"), ("band", "eps"),
                                       ("band", "nu"), ("hold", "nu")])
def test_rhs_vjp_params(orc, case, kind, name):
    g, u, rng = case
    rhs = orc.make_ns_rhs(g)
    v = _rc(rng, u.shape)
    base = {"nu": 0.02, "A": 0.3, "eps": 0.1}
    _, pb = orc.rhs_vjp(g, u, _params(orc, kind, **base), v)
    h = 1e-6
    up = dict(base, **{name: base[name] + h})
    dn = dict(base, **{name: base[name] - h})
    fd = (orc._dot_re(v, rhs(u, _params(orc, kind, **up), 0.0))
          - orc._dot_re(v, rhs(u, _params(orc, kind, **dn), 0.0))) / (2 * h)
    assert abs(pb[name] - fd) <= 1e-6 * max(abs(fd), 1e-3)


@pytest.mark.parametrize("kind", ["linear", "band", "hold"])
def test_rk4_step_vjp(orc, case, kind):
    g, u, rng = case
    p = _params(orc, kind)
    rhs = orc.make_ns_rhs(g)
    dt = 5e-3
    v, d = _rc(rng, u.shape), _rc(rng, u.shape)
    ub, pb = orc.rk4_step_vjp(g, u, p, dt, v)
    h = 1e-6
    fd = (orc._dot_re(v, orc.rk4_step(rhs, u + h * d, p, dt, 0.0))
          - orc._dot_re(v, orc.rk4_step(rhs, u - h * d, p, dt, 0.0))) / (2 * h)
    assert abs(orc._dot_re(ub, d) - fd) <= 1e-7 * abs(fd)


def test_rollout_vjp_checkpoints(orc, case):
    g, u, rng = case
    p = _params(orc, "linear", A=0.0)
    rhs = orc.make_ns_rhs(g)
    dt, n = 5e-3, 5
    v, d = _rc(rng, u.shape), _rc(rng, u.shape)
    ub, pb = orc.rollout_vjp(g, u, p, dt, n, v, checkpoint_every=2)
    ub1, pb1 = orc.rollout_vjp(g, u, p, dt, n, v)
    assert np.allclose(ub, ub1, rtol=1e-12, atol=0) and abs(pb["A"] - pb1["A"]) <= 1e-12 * abs(pb1["A"])
    h = 1e-6
    fd = (orc._dot_re(v, orc.rollout(rhs, u + h * d, p, dt, n)) - orc._dot_re(v, orc.rollout(rhs, u - h * d, p, dt, n))) / (2 * h)
    assert abs(orc._dot_re(ub, d) - fd) <= 1e-7 * abs(fd)
    pA = lambda A: orc.NSParams(nu=0.02, forcing=orc.LinearForcing(A))
    fdA = (orc._dot_re(v, orc.rollout(rhs, u, pA(h), dt, n)) - orc._dot_re(v, orc.rollout(rhs, u, pA(-h), dt, n))) / (2 * h)
    assert abs(pb["A"] - fdA) <= 1e-6 * abs(fdA)
