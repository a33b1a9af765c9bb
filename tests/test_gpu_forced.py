"""External force held over an RHS call or a rollout (``hit_rhs_forced``,
``hit_rollout_forced``; no reference counterpart -- the coarse-LES subgrid
term), the fused LES step built on it, and rollouts captured into the
caller's CUDA graph.

Tolerances (relative L2): float32 1e-5, float64 1e-12; a captured rollout is
bit-identical to the graph-replayed one (same kernels in the same order)."""

import importlib

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def _force(orc, og, seed):
    rng = np.random.default_rng(seed)
    dims = (og.Nx, og.Ny, og.Nz)
    # a force with modes outside the 2/3 box and a divergent part: the RHS
    # must mask and project it
    return 0.3 * orc.to_spectral(rng.standard_normal((3,) + dims).astype(og.dtype), og) / np.prod(dims) ** 0.5


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("dealiased", [True, False])
def test_rhs_and_rollout_with_external_force(h3, orc, dtype, dealiased):
    og = orc.make_grid(32, dtype=dtype)
    g = h3.make_grid(32, dtype=torch.float32 if dtype == np.float32 else torch.float64)
    u0 = orc.hit_initial_field(0, og)
    f = _force(orc, og, 1).astype(og.cdtype)
    nu = 0.02
    op = orc.NSParams(nu=nu, forcing=orc.BandForcing(0.1, 1.0, 2.0))
    p = h3.NSParams(nu=nu, forcing=h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0))
    orhs = orc.make_ns_rhs(og)
    pf = orc.project(orc.dealias(f, og), og)

    def orhs_f(u, prm, t):
        return orhs(u, prm, t) + pf

    tol = 1e-5 if dtype == np.float32 else 1e-12
    rhs = h3.make_ns_rhs(g)
    fd = torch.as_tensor(f).cuda()
    du = rhs(u0, p, 0.0, assume_dealiased=dealiased, f_ext=fd)
    assert rel_l2(_np(du), orhs_f(u0, op, 0.0)) < tol
    u = h3.rollout(rhs, u0, p, 2e-3, 3, assume_dealiased=dealiased, f_ext=fd)
    assert rel_l2(_np(u), orc.rollout(orhs_f, u0, op, 2e-3, 3)) < tol
    # the step graphs without the force are rebuilt after the forced ones
    u_free = h3.rollout(rhs, u0, p, 2e-3, 3, assume_dealiased=dealiased)
    assert rel_l2(_np(u_free), orc.rollout(orhs, u0, op, 2e-3, 3)) < tol


def test_rollout_captured_into_a_caller_graph_is_bit_identical(h3, orc):
    og = orc.make_grid(32, dtype=np.float32)
    g = h3.make_grid(32)
    u0 = torch.as_tensor(orc.hit_initial_field(2, og)).cuda()
    p = h3.NSParams(nu=0.02, forcing=h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0))
    rhs = h3.make_ns_rhs(g)
    ref = h3.rollout(rhs, u0, p, 2e-3, 3, assume_dealiased=True)
    static = u0.clone()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        h3.rollout(rhs, static, p, 2e-3, 3, assume_dealiased=True)
    torch.cuda.current_stream().wait_stream(s)
    gph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(gph):
        out = h3.rollout(rhs, static, p, 2e-3, 3, assume_dealiased=True)
    gph.replay()
    torch.cuda.synchronize()
    assert torch.equal(out, ref)


def test_fused_les_step_matches_composed_les_rhs(h3):
    les = importlib.import_module("3dhit_b200.les")
    closure_mod = importlib.import_module("3dhit_b200.closure")
    g = h3.make_grid(32)
    u0 = h3.hit_initial_field(3, g)
    nu = 0.01
    p = h3.NSParams(nu=nu, forcing=h3.HoldEnergyForcing(E_target=1.5, nu=nu, tau=0.5))
    cl = closure_mod.ClosureMLP(g.device, seed=1)
    cl.x_scale.fill_(5.0)
    cl.y_scale.fill_(2.0)
    dt = 2e-3
    a = les.FusedLESStep(g, cl, p, dt)(u0)
    b = h3.rk4_step(les.LESRHS(g, cl, freeze_every=4), u0, p, dt, 0.0)
    c = h3.rk4_step(les.LESRHS(g, None), u0, p, dt, 0.0)
    assert rel_l2(_np(a), _np(b)) < 1e-5
    assert rel_l2(_np(a), _np(c)) > 1e-4  # the closure does act
    assert rel_l2(_np(les.FusedLESStep(g, None, p, dt)(u0)), _np(c)) < 1e-5


def test_lagged_les_step_uses_the_previous_state_force(h3):
    les = importlib.import_module("3dhit_b200.les")
    closure_mod = importlib.import_module("3dhit_b200.closure")
    g = h3.make_grid(32)
    u0 = h3.hit_initial_field(4, g)
    nu = 0.01
    p = h3.NSParams(nu=nu, forcing=h3.HoldEnergyForcing(E_target=1.5, nu=nu, tau=0.5))
    cl = closure_mod.ClosureMLP(g.device, seed=2)
    cl.x_scale.fill_(5.0)
    cl.y_scale.fill_(2.0)
    dt = 2e-3
    lagged = les.FusedLESStep(g, cl, p, dt, lag=True)
    plain = les.FusedLESStep(g, cl, p, dt)
    u1 = lagged(u0)
    assert torch.equal(u1, plain(u0))  # the first step uses its own state's force
    u2 = lagged(u1)
    f0 = plain.force(u0).clone()
    ref = h3.rk4_step(h3.make_ns_rhs(g), u1, p, dt, 0.0, assume_dealiased=True, f_ext=f0)
    torch.cuda.synchronize()
    assert torch.equal(u2, ref)
