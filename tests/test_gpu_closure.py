"""Tensor-core (tcgen05) kernels of the learned subgrid-stress closure against
torch float32 references of the same operations (bf16 operands are exact in
float32; only the accumulation order differs)."""
import importlib

import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nat():
    return importlib.import_module("3dhit_b200._native")


@pytest.mark.parametrize("M,N,K", [(300, 64, 80), (128, 16, 16), (1000, 128, 64), (257, 32, 144)])
def test_tc_gemm_bf16(nat, M, N, K):
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C = torch.full((M, N), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    nat.call("hit_tc_gemm_bf16", nat.ptr(A), K, nat.ptr(B), K, nat.ptr(C), N, M, N, K, nat.ptr(err),
             nat.stream_ptr(A.device))
    ref = A.float() @ B.float().T
    assert int(err.item()) == 0
    assert torch.allclose(C, ref, rtol=1e-5, atol=1e-4 * float(ref.abs().max()))


def _mlp_case(h3mod, P, seed):
    closure = importlib.import_module("3dhit_b200.closure")
    m = closure.ClosureMLP("cuda", seed=seed)
    g = torch.Generator().manual_seed(seed + 1)
    x = torch.randn(P, 9, generator=g) * 1.5
    tau = torch.randn(P, 6, generator=g) * 0.5
    return m, x, tau


def _np_params(m):
    return [t.detach().cpu().numpy() for t in m.params]


def test_mlp_forward_matches_oracle(h3, orc):
    m, x, tau = _mlp_case(h3, 1000, 3)
    y = m.raw_forward(x.cuda()).cpu().numpy()
    yo, _, _ = orc.mlp_loss_grads(_np_params(m), x.numpy(), tau.numpy())
    m.check_errors()
    import numpy as np
    assert np.linalg.norm(y - yo) <= 1e-3 * np.linalg.norm(yo)


def test_mlp_grads_match_oracle(h3, orc):
    """Loss and all eight parameter gradients of the tensor-core training pass
    against the oracle restatement with the same bf16 roundings."""
    import numpy as np
    m, x, tau = _mlp_case(h3, 4096, 5)
    loss = float(m.loss_and_grads(x.cuda(), tau.cuda()).item())
    m.check_errors()
    _, lo, go = orc.mlp_loss_grads(_np_params(m), x.numpy(), tau.numpy())
    assert abs(loss - lo) <= 1e-4 * lo
    for p, ref in zip(m.params, go):
        got = p.grad.cpu().numpy().astype(np.float64)
        assert np.linalg.norm(got - ref) <= 1e-2 * np.linalg.norm(ref), (got.shape, np.linalg.norm(got - ref) / np.linalg.norm(ref))


def test_mlp_grads_close_to_float32_autograd(h3):
    """Against torch autograd of the same network in float32 (no bf16): equal
    to the bf16 rounding of weights and activations."""
    m, x, tau = _mlp_case(h3, 4096, 7)
    m.loss_and_grads(x.cuda(), tau.cuda())
    ps = [p.detach().clone().requires_grad_(True) for p in m.params]
    W1, b1, W2, b2, W3, b3, W4, b4 = ps
    def gelu(v):
        return torch.nn.functional.gelu(v, approximate="tanh")
    xc, tc_ = x.cuda(), tau.cuda()
    y = gelu(gelu(gelu(xc @ W1 + b1) @ W2 + b2) @ W3 + b3) @ W4 + b4
    loss = ((y - tc_) ** 2).mean()
    loss.backward()
    for p, q in zip(m.params, ps):
        assert torch.linalg.vector_norm(p.grad - q.grad) <= 5e-2 * torch.linalg.vector_norm(q.grad)


def test_mlp_training_reduces_loss(h3):
    """A few Adam steps on the tensor-core gradients fit a smooth target."""
    closure = importlib.import_module("3dhit_b200.closure")
    m = closure.ClosureMLP("cuda", seed=11)
    g = torch.Generator().manual_seed(12)
    x = (torch.randn(8192, 9, generator=g)).cuda()
    tau = torch.stack([x[:, 0] * x[:, 4], x[:, 1] + x[:, 3], x[:, 8] ** 2, torch.tanh(x[:, 2]), x[:, 5] * 0.5,
                       x[:, 6] - x[:, 7]], 1) * 0.3
    for p in m.params:
        p.requires_grad_(True)
    opt = torch.optim.Adam(m.params, lr=3e-3)
    losses = []
    for it in range(300):
        losses.append(float(m.loss_and_grads(x, tau).item()))
        opt.step()
        m.pack()
    m.check_errors()
    assert losses[-1] < 0.2 * losses[0], (losses[0], losses[-1])


def test_les_pieces_against_torch(h3):
    """Velocity gradients, the SGS force and the box filter of the LES path
    against torch references of the same spectral formulas."""
    les = importlib.import_module("3dhit_b200.les")
    g = h3.make_grid(32, dtype=torch.float64)
    u = h3.random_field(3, g)
    # gradients: irfftn(1j k_j u_i)
    grads = les.velocity_gradients(u, g)
    ks = [g.kx, g.ky, g.kz]
    ref = torch.stack([h3.to_physical(1j * ks[j] * u[i], g).reshape(-1) for i in range(3) for j in range(3)])
    assert torch.allclose(grads, ref, rtol=0, atol=1e-12 * float(ref.abs().max()))
    # SGS force: du += project(dealias(-1j k_j tau_ij))
    tau = torch.randn(6, 32, 32, 32, dtype=torch.float64, device="cuda")
    th = h3.to_spectral(tau, g)
    du = torch.zeros_like(u)
    import importlib as il
    nat = il.import_module("3dhit_b200._native")
    nat.call("hit_add_sgs_force", g.plan.handle, nat.ptr(th), nat.ptr(du), nat.stream_ptr(g.device))
    T = [[th[0], th[3], th[4]], [th[3], th[1], th[5]], [th[4], th[5], th[2]]]
    f = torch.stack([-1j * (ks[0] * T[i][0] + ks[1] * T[i][1] + ks[2] * T[i][2]) for i in range(3)])
    refd = h3.project(h3.dealias(f, g), g)
    assert torch.allclose(du, refd, rtol=0, atol=1e-12 * float(refd.abs().max()))
    # box filter of a field inside the coarse box: the same physical field at the coarse points
    gf = h3.make_grid(32, dtype=torch.float64)
    gc = h3.make_grid(16, dtype=torch.float64)
    uf = h3.random_field(4, gf)
    uc = les.box_filter(uf, gf, gc)
    xf = h3.to_physical(h3.dealias(uf * (torch.sqrt(gf.k2) <= 5).to(uf.dtype), gf), gf)
    uc5 = les.box_filter(h3.dealias(uf * (torch.sqrt(gf.k2) <= 5).to(uf.dtype), gf), gf, gc)
    xc = h3.to_physical(uc5, gc)
    assert torch.allclose(xc, xf[:, ::2, ::2, ::2], rtol=0, atol=1e-12 * float(xf.abs().max()))
    assert uc.shape == (3, 16, 16, 9)


def test_les_rhs_and_closure_smoke(h3):
    """LESRHS without a closure is the Navier-Stokes RHS; with an (untrained)
    closure it adds a finite, dealiased, divergence-free SGS force."""
    les = importlib.import_module("3dhit_b200.les")
    closure = importlib.import_module("3dhit_b200.closure")
    g = h3.make_grid(32)
    u = h3.hit_initial_field(0, g)
    p = h3.NSParams(nu=0.01, forcing=h3.LinearForcing(0.1))
    base = h3.make_ns_rhs(g)(u, p, 0.0)
    assert torch.equal(les.LESRHS(g)(u, p, 0.0), base)
    m = closure.ClosureMLP("cuda", seed=1)
    du = les.LESRHS(g, m)(u, p, 0.0)
    f = du - base
    assert torch.isfinite(f).all() and float(f.abs().max()) > 0
    assert torch.equal(f, h3.dealias(f, g))
    div = g.kx * f[0] + g.ky * f[1] + g.kz * f[2]
    assert float(div.abs().max()) <= 1e-4 * float(f.abs().max()) * float(g.k2.max()) ** 0.5
