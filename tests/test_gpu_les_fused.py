"""The learned closure fused into the coarse-LES step's own passes
(`hit_les_rollout`, `FusedLESStep(fused=True)`) against the same scheme
composed from separate calls (`FusedLESStep(fused=False)`: velocity
gradients, the MLP, rfftn of the stresses, the SGS force held over the four
stages of one fused RK4 step).  Both evaluate the closure once per step at
the step's initial state; they differ only in rounding (the fused path forms
the gradients, u x w and the force inside its transforms, and the MLP rounds
its inputs to bf16).  The closure is a seeded network with its inputs
scaled by the gradients' RMS; its force changes the step by more than
the tolerance on the state, and the closure's share of the step is
compared on its own."""

import importlib

import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _setup(h3, n, seed=1):
    cl = importlib.import_module("3dhit_b200.closure")
    nat = h3._native
    g = h3.make_grid(n)
    u0 = h3.hit_initial_field(0, g)
    grads = torch.empty(9, n ** 3, device=g.device)
    nat.call("hit_velocity_gradients", g.plan.handle, nat.ptr(u0), nat.ptr(grads), nat.stream_ptr(g.device))
    model = cl.ClosureMLP(g.device, seed=seed)
    model.x_scale = grads.std(dim=1).contiguous()
    model.y_scale = torch.full((6,), 0.5, device=g.device)
    p = h3.NSParams(nu=0.01, forcing=h3.HoldEnergyForcing(float(h3.energy(u0, g)), 0.01, tau=0.5))
    return g, u0, model, p


def _np(t):
    return t.cpu().numpy()


@pytest.mark.parametrize("n", [32, 64])
def test_fused_les_step_matches_composed(h3, n):
    les = importlib.import_module("3dhit_b200.les")
    g, u0, model, p = _setup(h3, n)
    dt = 2e-3
    composed = les.FusedLESStep(g, model, p, dt, fused=False)
    fused = les.FusedLESStep(g, model, p, dt, fused=True)
    plain = les.FusedLESStep(g, None, p, dt)
    u_c, u_f, u_0 = composed(u0), fused(u0), plain(u0)
    torch.cuda.synchronize()
    model.check_errors()
    h3.check_device("fused LES step")
    effect = rel_l2(_np(u_c), _np(u_0))
    assert effect > 1e-5, effect  # the closure's force changes the step
    # the closure's contribution to the step agrees to 0.2%, the state to 1e-5
    assert rel_l2(_np(u_f - u_0), _np(u_c - u_0)) < 2e-3
    assert rel_l2(_np(u_f), _np(u_c)) < 1e-5
    # several steps in one call (the device loop) against step-by-step composed
    nsteps = 5
    x = u0
    for _ in range(nsteps):
        x = composed(x)
    nat = h3._native
    out = torch.empty_like(u0)
    prm = h3.forcing.native_params(p.nu, p.forcing, nat.HIT_FLAG_ASSUME_DEALIASED)
    cl = importlib.import_module("3dhit_b200.closure")
    nat.call("hit_les_rollout", g.plan.handle, nat.ptr(u0), prm, cl.ctypes_ref(model._physical[0]), dt, nsteps,
             nat.ptr(out), nat.ptr(model._err), nat.stream_ptr(g.device))
    torch.cuda.synchronize()
    model.check_errors()
    assert rel_l2(_np(out), _np(x)) < 3e-5


def test_fused_les_step_rejects_what_it_does_not_cover(h3):
    nat = h3._native
    cl = importlib.import_module("3dhit_b200.closure")
    g = h3.make_grid(32, 32, 16)  # Nz = 16: no fused z pass at this length
    u0 = h3.hit_initial_field(0, g)
    model = cl.ClosureMLP(g.device)
    model.pack_physical()
    p = h3.NSParams(nu=0.01)
    prm = h3.forcing.native_params(p.nu, p.forcing, nat.HIT_FLAG_ASSUME_DEALIASED)
    lib = nat.load()
    rc = lib.hit_les_rollout(g.plan.handle, nat.ptr(u0), prm, cl.ctypes_ref(model._physical[0]), 1e-3, 1,
                             nat.ptr(torch.empty_like(u0)), nat.ptr(model._err), nat.stream_ptr(g.device))
    assert rc == nat.HIT_E_UNSUPPORTED
    assert b"Nz in {32, 64, 128}" in lib.hit_last_error_string()
