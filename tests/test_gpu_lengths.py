"""Every transform length of the CUDA path (64 ... 1024 points) along each
axis in turn, against the oracle: the RHS and one RK4 step on
(N, 16, 16), (16, N, 16) and (16, 16, N) grids.  The x and y transforms,
the register-mode x-forward epilogue (512-point float columns) and the z pass
(N/2-point complex transforms) all run at the lengths of the 512^3 and
1024^3 workloads here, on grids the oracle finishes in milliseconds.

Tolerances (relative L2): float32 1e-5, float64 1e-12."""

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

LENGTHS = (64, 128, 256, 512, 1024)


def _dims(axis, n):
    d = [16, 16, 16]
    d[axis] = n
    return tuple(d)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("n", LENGTHS)
def test_rhs_and_step_at_every_length(h3, orc, n, axis, dtype):
    dims = _dims(axis, n)
    og = orc.make_grid(*dims, dtype=dtype)
    g = h3.make_grid(*dims, dtype=torch.float32 if dtype == np.float32 else torch.float64)
    rng = np.random.default_rng(n + 7 * axis)
    u0 = orc.to_spectral(rng.standard_normal((3,) + dims).astype(dtype), og)
    u0 = orc.project(orc.dealias(u0, og), og).astype(og.cdtype)
    f = orc.BandForcing(eps=0.1, kmin=1.0, kmax=2.0)
    op = orc.NSParams(nu=0.01, forcing=f)
    p = h3.NSParams(nu=0.01, forcing=h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0))
    tol = 1e-5 if dtype == np.float32 else 1e-12
    rhs, orhs = h3.make_ns_rhs(g), orc.make_ns_rhs(og)
    du0 = orhs(u0, op, 0.0)
    u1o = orc.rk4_step(orhs, u0, op, 1e-3, 0.0)
    for dealiased in (True, False):
        du = rhs(u0, p, 0.0, assume_dealiased=dealiased)
        assert rel_l2(du.cpu().numpy(), du0) < tol, ("rhs", dealiased)
        u1 = h3.rk4_step(rhs, u0, p, 1e-3, 0.0, assume_dealiased=dealiased)
        assert rel_l2(u1.cpu().numpy(), u1o) < tol, ("step", dealiased)
