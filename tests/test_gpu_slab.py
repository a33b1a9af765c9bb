"""The CUDA side of the slab-decomposed RHS on one GPU: the per-axis
transforms (``hit_axis_fft``) against torch.fft, and the slab RHS with one
rank (its exchanges are copies) against the package's RHS.  The two-rank
partition and exchanges are tested on the CPU (tests/test_multirank_slab.py)."""

import importlib

import pytest
import torch

pytestmark = pytest.mark.gpu

slab = importlib.import_module("3dhit_b200.slab")


def _rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


@pytest.mark.parametrize("dtype,tol", [(torch.float32, 2e-6), (torch.float64, 1e-13)])
def test_axis_transforms_match_torch_fft(dtype, tol):
    lay = slab.SlabLayout(16, 32, 64, 1, 0)
    T = slab.CudaSlabTransforms(lay, 6.28, 6.28, 6.28, dtype, "cuda")
    gen = torch.Generator(device="cuda").manual_seed(0)
    r = torch.randn(2, 16, 32, 64, generator=gen, device="cuda", dtype=dtype)
    c = torch.fft.rfft(r, dim=3)
    assert _rel(T.z_r2c(r), c) < tol
    assert _rel(T.z_c2r(c), torch.fft.irfft(c, n=64, dim=3, norm="forward")) < tol
    assert _rel(T.x(c, True), torch.fft.ifft(c, dim=1, norm="forward")) < tol
    assert _rel(T.x(c, False), torch.fft.fft(c, dim=1)) < tol
    assert _rel(T.y(c, True), torch.fft.ifft(c, dim=2, norm="forward")) < tol
    assert _rel(T.y(c, False), torch.fft.fft(c, dim=2)) < tol


@pytest.mark.parametrize("dtype,tol", [(torch.float32, 1e-5), (torch.float64, 1e-12)])
def test_single_rank_slab_rhs_matches_package_rhs(h3, dtype, tol):
    g = h3.make_grid(32, 16, 32, dtype=dtype)
    u0 = h3.hit_initial_field(0, g)
    rhs = slab.SlabRHS(32, 16, 32, dtype=dtype)
    for f in (h3.NoForcing(), h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0)):
        p = h3.NSParams(nu=0.02, forcing=f)
        ref = h3.make_ns_rhs(g)(u0, p, 0.0, assume_dealiased=False)
        assert _rel(rhs(u0, p), ref) < tol
