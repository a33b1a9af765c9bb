"""cuFFT (through torch.fft on the GPU) as a correctness check of the
hand-written transforms and of the fused RHS: the reference's RHS
(src/hit3d/navierstokes.py:62-97) composed from torch ops and cuFFT
irfftn/rfftn (the numpy/XLA axis convention of src/hit3d/grid.py:181-188)
against the fused kernels.  cuFFT is not on the product path.

Tolerances (relative L2): float32 1e-5, float64 1e-12."""

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

DIMS = [(64, 64, 64), (32, 64, 128), (128, 32, 16), (16, 16, 1024), (16, 8, 4)]


def _tol(dtype):
    return 1e-5 if dtype == torch.float32 else 1e-12


def cufft_rhs(u_hat, g, nu, A):
    """The reference's RHS with a LinearForcing(A), from torch ops and cuFFT."""
    s, dims = (g.Nx, g.Ny, g.Nz), (1, 2, 3)
    kx, ky, kz = g.kx, g.ky, g.kz
    w_hat = 1j * torch.stack((ky * u_hat[2] - kz * u_hat[1], kz * u_hat[0] - kx * u_hat[2],
                              kx * u_hat[1] - ky * u_hat[0]))
    u = torch.fft.irfftn(u_hat, s=s, dim=dims)
    w = torch.fft.irfftn(w_hat, s=s, dim=dims)
    nl = torch.stack((u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]))
    du = (torch.fft.rfftn(nl, dim=dims) + A * u_hat) * g.dealias
    div = (kx * du[0] + ky * du[1] + kz * du[2]) * g.inv_k2
    du = du - torch.stack((kx * div, ky * div, kz * div))
    return du - nu * g.k2 * u_hat


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("dims", DIMS)
def test_transforms_and_rhs_match_cufft(h3, dims, dtype):
    g = h3.make_grid(*dims, dtype=dtype)
    gen = torch.Generator(device="cuda").manual_seed(sum(dims))
    u = torch.randn((3,) + dims, generator=gen, dtype=dtype, device="cuda")
    s, ax = dims, (1, 2, 3)
    uh = h3.to_spectral(u, g)
    assert rel_l2(uh.cpu().numpy(), torch.fft.rfftn(u, dim=ax).cpu().numpy()) < _tol(dtype)
    back = h3.to_physical(uh, g)
    assert rel_l2(back.cpu().numpy(), torch.fft.irfftn(uh, s=s, dim=ax).cpu().numpy()) < _tol(dtype)
    u0 = h3.project(h3.dealias(uh, g), g) / float(np.prod(dims)) ** 0.5
    nu, A = 0.01, 0.1333
    du = h3.make_ns_rhs(g)(u0, h3.NSParams(nu=nu, forcing=h3.LinearForcing(A=A)), 0.0)
    assert rel_l2(du.cpu().numpy(), cufft_rhs(u0, g, nu, A).cpu().numpy()) < _tol(dtype)
