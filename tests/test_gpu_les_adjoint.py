"""Discrete adjoint of the coarse LES step with the learned closure.

Each transpose is checked on its own: the SGS force and the velocity
gradients by the dot-product identity <A x, y> = <x, A^T y> in float64
(cotangents: dL/dRe + i dL/dIm of stored spectral entries, so the spectral
inner product is sum Re(conj(a) b)); the RK4 step with a held force by central
finite differences in float64 (both the state's and the force's cotangent,
with the hold-energy forcing's chain rule); the MLP's vector-Jacobian product
against float32 autograd of the same bf16-weighted network.  The whole LES
window gradient (all of them chained) is checked by descent: a small step
against it lowers the spectrum loss."""

import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

les = importlib.import_module("3dhit_b200.les")
cl = importlib.import_module("3dhit_b200.closure")
fmod = importlib.import_module("3dhit_b200.forcing")


def _re_dot(a, b):
    return float(torch.sum(a.real * b.real + a.imag * b.imag))


def _spectral_of_real(h3, g, nc, seed):
    gen = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.randn(nc, g.Nx, g.Ny, g.Nz, generator=gen, device="cuda", dtype=g.dtype)
    return h3.to_spectral(x, g)


def test_sgs_force_transpose_dot_product(h3):
    nat = h3._native
    g = h3.make_grid(16, 16, 32, dtype=torch.float64)
    P = g.Nx * g.Ny * g.Nz
    gen = torch.Generator(device="cuda").manual_seed(1)
    tau = torch.randn(6, g.Nx, g.Ny, g.Nz, generator=gen, device="cuda", dtype=torch.float64)
    f = torch.empty(3, g.Nx, g.Ny, g.Nz // 2 + 1, dtype=torch.complex128, device="cuda")
    tau_hat = h3.to_spectral(tau, g)
    nat.call("hit_sgs_force", g.plan.handle, nat.ptr(tau_hat), nat.ptr(f), nat.stream_ptr(g.device))
    fb = _spectral_of_real(h3, g, 3, 2)
    tb = torch.empty(6, P, dtype=torch.float64, device="cuda")
    nat.call("hit_sgs_force_vjp", g.plan.handle, nat.ptr(fb), nat.ptr(tb), nat.stream_ptr(g.device))
    lhs = _re_dot(f, fb)
    rhs = float(torch.sum(tau.reshape(6, -1) * tb))
    assert abs(lhs - rhs) < 1e-11 * max(abs(lhs), 1e-300), (lhs, rhs)


def test_velocity_gradients_transpose_dot_product(h3):
    nat = h3._native
    g = h3.make_grid(32, 16, 16, dtype=torch.float64)
    u = _spectral_of_real(h3, g, 3, 3)
    gr = les.velocity_gradients(u, g)
    gen = torch.Generator(device="cuda").manual_seed(4)
    gb = torch.randn(gr.shape, generator=gen, device="cuda", dtype=torch.float64)
    ub = torch.zeros_like(u)
    nat.call("hit_velocity_gradients_vjp", g.plan.handle, nat.ptr(gb), nat.ptr(ub), nat.stream_ptr(g.device))
    lhs = float(torch.sum(gr * gb))
    rhs = _re_dot(u, ub)
    assert abs(lhs - rhs) < 1e-11 * max(abs(lhs), 1e-300), (lhs, rhs)


@pytest.mark.parametrize("forcing", ["hold", "band"])
def test_forced_step_transpose_finite_differences(h3, forcing):
    nat = h3._native
    g = h3.make_grid(16, dtype=torch.float64)
    nu = 0.02
    f_obj = (fmod.HoldEnergyForcing(1.5, nu) if forcing == "hold" else h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0))
    p = h3.NSParams(nu=nu, forcing=f_obj)
    rhs = h3.make_ns_rhs(g)
    u = h3.hit_initial_field(0, g)
    un = float(torch.linalg.vector_norm(u))

    def scaled(v, s):  # v with norm s |u|
        return v * (s * un / float(torch.linalg.vector_norm(v)))

    f = scaled(h3.dealias_project(_spectral_of_real(h3, g, 3, 5), g), 0.1)
    dt = 2e-3
    ct = h3.random_field(6, g)
    ub = torch.empty_like(u)
    fb = torch.empty_like(u)
    prm = fmod.native_params(nu, f_obj, 0)
    nat.call("hit_rk4_step_forced_vjp", g.plan.handle, nat.ptr(u), prm, nat.ptr(f), dt, 0.0, nat.ptr(ct),
             nat.ptr(ub), nat.ptr(fb), None, nat.stream_ptr(g.device))
    # directions as large as the state, so that the differences stay far
    # above the float64 rounding of the (large) inner product
    du = scaled(h3.random_field(7, g), 1.0)
    df = scaled(h3.random_field(8, g), 1.0)

    def L(uu, ff):
        return _re_dot(ct, h3.rk4_step(rhs, uu, p, dt, 0.0, assume_dealiased=False, f_ext=ff))

    h = 1e-4  # truncation ~h^2, rounding of the inner product ~1e-16 |L| / h: both near 1e-8
    fd_u = (L(u + h * du, f) - L(u - h * du, f)) / (2 * h)
    fd_f = (L(u, f + h * df) - L(u, f - h * df)) / (2 * h)
    assert _re_dot(ub, du) == pytest.approx(fd_u, rel=1e-6)
    assert _re_dot(fb, df) == pytest.approx(fd_f, rel=1e-6)


def test_mlp_vjp_matches_autograd(h3):
    m = cl.ClosureMLP(torch.device("cuda"), seed=3)
    m.x_scale = torch.rand(9, device="cuda") + 0.5
    m.y_scale = torch.rand(6, device="cuda") + 0.5
    m.sgs_scale = 0.8
    P = 128 * 40
    gen = torch.Generator(device="cuda").manual_seed(9)
    x = torch.randn(9, P, generator=gen, device="cuda")
    yb = torch.randn(6, P, generator=gen, device="cuda")
    xbar, grads = m.vjp(x, yb)
    m.check_errors()
    # float32 autograd of the network with bf16-rounded operands
    params = [q.detach().clone().requires_grad_(True) for q in m.params]
    W1, b1, W2, b2, W3, b3, W4, b4 = params
    xs = x.T.clone().requires_grad_(True)
    bf = lambda t: t.to(torch.bfloat16).float()  # noqa: E731
    gelu = lambda z: 0.5 * z * (1 + torch.tanh(0.7978845608028654 * (z + 0.044715 * z ** 3)))  # noqa: E731
    a1 = bf(gelu(bf(xs) @ bf(W1 / m.x_scale[:, None]) + bf(b1)))
    a2 = bf(gelu(a1 @ bf(W2) + b2))
    a3 = bf(gelu(a2 @ bf(W3) + b3))
    ys = m.y_scale * m.sgs_scale
    y = a3 @ bf(W4 * ys) + b4 * ys
    (y * yb.T).sum().backward()
    for got, q in zip(grads, params):
        err = float(torch.linalg.vector_norm(got - q.grad) / torch.linalg.vector_norm(q.grad))
        assert err < 5e-2, err
    err = float(torch.linalg.vector_norm(xbar.T - xs.grad) / torch.linalg.vector_norm(xs.grad))
    assert err < 5e-2, err


def test_les_window_gradient_is_a_descent_direction(h3):
    """Chained transposes through 12 LES steps (32^3, hold-energy forcing,
    closure on): stepping the master parameters, or the initial state, a
    little against the gradient lowers the spectrum loss."""
    g = h3.make_grid(32)
    u0 = h3.hit_initial_field(1, g)
    m = cl.ClosureMLP(torch.device("cuda"), seed=1)
    gr = les.velocity_gradients(u0, g)
    m.x_scale = gr.std(1)
    m.y_scale = torch.full((6,), float(gr.std()) ** 2 * 2e-3, device="cuda")
    p = h3.NSParams(nu=0.02, forcing=fmod.HoldEnergyForcing(1.5, 0.02, tau=0.5))
    dt = h3.cfl_dt(u0, g, 0.5)
    _, E = h3.energy_spectrum(u0, g)
    logT = torch.log(torch.as_tensor(E[:10], device="cuda") * 1.3)

    def loss(u):
        return les.spectrum_log_loss(u, g, logT)

    step = les.FusedLESStep(g, m, p, dt)
    L0, grads, ub, _ = les.les_window_grad(step, u0, 12, loss)
    norm = float(torch.sqrt(sum((d.double() ** 2).sum() for d in grads)))
    assert np.isfinite(L0) and norm > 0
    saved = [q.clone() for q in m.params]
    eta = 1e-2 / norm
    for q, d in zip(m.params, grads):
        q -= eta * d
    m._packed = m._physical = None
    L1, _, _, _ = les.les_window_grad(les.FusedLESStep(g, m, p, dt), u0, 12, loss)
    for q, s in zip(m.params, saved):
        q.copy_(s)
    m._packed = m._physical = None
    e = 1e-2 * float(torch.linalg.vector_norm(u0)) / float(torch.linalg.vector_norm(ub))
    L2, _, _, _ = les.les_window_grad(les.FusedLESStep(g, m, p, dt), u0 - e * ub, 12, loss)
    print(f"LES window loss {L0:.6f}: params step {L1:.6f}, state step {L2:.6f}")
    assert L1 < L0 and L2 < L0
