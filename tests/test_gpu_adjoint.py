"""The CUDA discrete adjoint (hit_rhs_vjp / hit_rk4_step_vjp / hit_rollout_vjp)
against the oracle's transpose (itself pinned by finite differences on the
CPU) and against central finite differences of the CUDA forward path.

The reference differentiates with jax.vjp (src/hit3d/navierstokes.py:62-97,
src/hit3d/integrators.py:32-53); cotangents here are dL/dRe + i dL/dIm of the
stored entries (PyTorch's convention, the complex conjugate of jax.vjp's).
Tolerances: float64 paths agree with the float64 oracle to 1e-10 relative
(both are exact transposes up to rounding); float32 paths to 2e-4 relative
L2 (float32 rounding of the forward and the transpose)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

FORCINGS = ["none", "linear", "band", "hold"]


def _rc(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _params(mod, kind, nu=0.02, A=0.3, eps=0.1, tau=0.7):
    f = {"none": mod.NoForcing(), "linear": mod.LinearForcing(A), "band": mod.BandForcing(eps, 1.0, 2.0),
         "hold": mod.HoldEnergyForcing(1.5, nu, tau=tau)}[kind]
    return mod.NSParams(nu=nu, forcing=f)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def case(h3, orc):
    dims = (16, 16, 8)
    og = orc.make_grid(*dims, dtype=np.float64)
    u = orc.random_field(5, og)
    rng = np.random.default_rng(11)
    return dims, og, u, rng


def _dev(x, dt=torch.complex128):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dt, device="cuda")


@pytest.mark.parametrize("kind", FORCINGS)
def test_rhs_vjp_matches_oracle_f64(h3, orc, case, kind):
    dims, og, u, rng = case
    g = h3.make_grid(*dims, dtype=torch.float64)
    v = _rc(rng, u.shape)
    ub, pb = h3.rhs_vjp(h3.make_ns_rhs(g), _dev(u), _params(h3, kind), _dev(v))
    ubo, pbo = orc.rhs_vjp(og, u, _params(orc, kind), v)
    assert _rel(ub.cpu().numpy(), ubo) < 1e-10
    for k in ("nu", "A", "eps"):
        assert abs(pb[k] - pbo.get(k, 0.0)) <= 1e-10 * max(1.0, abs(pbo.get(k, 0.0)))


@pytest.mark.parametrize("kind", ["linear", "band"])
def test_rhs_vjp_f32(h3, orc, case, kind):
    dims, og, u, rng = case
    g = h3.make_grid(*dims, dtype=torch.float32)
    v = _rc(rng, u.shape)
    ub, pb = h3.rhs_vjp(h3.make_ns_rhs(g), _dev(u, torch.complex64), _params(h3, kind), _dev(v, torch.complex64))
    ubo, pbo = orc.rhs_vjp(og, u, _params(orc, kind), v)
    assert _rel(ub.cpu().numpy().astype(np.complex128), ubo) < 2e-4


@pytest.mark.parametrize("kind", ["linear", "band", "hold"])
def test_rk4_step_vjp_matches_oracle_f64(h3, orc, case, kind):
    dims, og, u, rng = case
    g = h3.make_grid(*dims, dtype=torch.float64)
    v = _rc(rng, u.shape)
    dt = 5e-3
    ub, pb = h3.rk4_step_vjp(h3.make_ns_rhs(g), _dev(u), _params(h3, kind), dt, _dev(v))
    ubo, pbo = orc.rk4_step_vjp(og, u, _params(orc, kind), dt, v)
    assert _rel(ub.cpu().numpy(), ubo) < 1e-10
    for k in ("nu", "A", "eps"):
        assert abs(pb[k] - pbo.get(k, 0.0)) <= 1e-9 * max(1.0, abs(pbo.get(k, 0.0)))


def test_rollout_vjp_oracle_and_fd_f64(h3, orc, case):
    """Checkpoints every 3 of 7 steps; the gradient w.r.t. u0 and A against the
    oracle and against central differences of the CUDA rollout."""
    dims, og, u, rng = case
    g = h3.make_grid(*dims, dtype=torch.float64)
    rhs = h3.make_ns_rhs(g)
    dt, n = 5e-3, 7
    p = _params(h3, "linear", A=0.05)
    v = _rc(rng, u.shape)
    ub, pb = h3.rollout_vjp(rhs, _dev(u), p, dt, n, _dev(v), checkpoint_every=3)
    ubo, pbo = orc.rollout_vjp(og, u, _params(orc, "linear", A=0.05), dt, n, v, checkpoint_every=3)
    assert _rel(ub.cpu().numpy(), ubo) < 1e-10
    assert abs(pb["A"] - pbo["A"]) <= 1e-9 * abs(pbo["A"])
    assert abs(pb["nu"] - pbo["nu"]) <= 1e-9 * abs(pbo["nu"])

    def L(x, A=0.05):
        out = h3.rollout(rhs, _dev(x), _params(h3, "linear", A=A), dt, n, assume_dealiased=False)
        return float(np.sum(np.real(np.conj(v) * out.cpu().numpy())))

    h = 1e-6
    for s in range(3):
        d = _rc(np.random.default_rng(100 + s), u.shape)
        fd = (L(u + h * d) - L(u - h * d)) / (2 * h)
        ad = float(np.sum(np.real(np.conj(ub.cpu().numpy()) * d)))
        assert abs(ad - fd) <= 1e-7 * abs(fd)
    fdA = (L(u, 0.05 + h) - L(u, 0.05 - h)) / (2 * h)
    assert abs(pb["A"] - fdA) <= 1e-7 * abs(fdA)


def test_rollout_autograd(h3, orc, case):
    """torch autograd through rollout_autograd gives the adjoint's gradients."""
    dims, og, u, rng = case
    g = h3.make_grid(*dims, dtype=torch.float64)
    rhs = h3.make_ns_rhs(g)
    u0 = _dev(u).requires_grad_(True)
    A = torch.tensor(0.05, dtype=torch.float64, requires_grad=True)
    nu = torch.tensor(0.02, dtype=torch.float64, requires_grad=True)
    p = h3.NSParams(nu=nu, forcing=h3.LinearForcing(A))
    out = h3.rollout_autograd(rhs, u0, p, 5e-3, 4, checkpoint_every=2)
    loss = (out.abs() ** 2 * g.weights).sum()
    loss.backward()
    ct = (2 * g.weights * out.detach()).to(torch.complex128)
    ub, pb = h3.rollout_vjp(rhs, _dev(u), h3.NSParams(nu=0.02, forcing=h3.LinearForcing(0.05)), 5e-3, 4, ct,
                            checkpoint_every=2)
    # autograd forms the cotangent as 2|z| (z/|z|) w, the test as 2 w z: equal
    # to rounding, so compare against the norm
    assert float((u0.grad - ub).abs().max()) <= 1e-12 * float(ub.abs().max())
    assert abs(float(A.grad) - pb["A"]) <= 1e-10 * abs(pb["A"])
    assert abs(float(nu.grad) - pb["nu"]) <= 1e-10 * abs(pb["nu"])
