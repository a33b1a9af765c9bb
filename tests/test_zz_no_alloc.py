"""hit_energy_spectrum_noalloc: the spectrum entry point for callers that
cannot allocate device memory (code inside CUDA stream capture, an XLA custom
call that gets every buffer from XLA, a process whose memory another allocator
has reserved).  Its scratch is a static device array shared by all calls, so
it is checked against the plan-based hit_energy_spectrum on two calls in a
row with different inputs: the second call must not see the first call's
partial sums.  Collected last so that a failure here comes after every other
test has run."""

import ctypes
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _noalloc(nat, g, u):
    ns = g.plan.num_shells
    E = torch.full((ns,), float("nan"), dtype=torch.float64, device=g.device)
    Ec = torch.full((3 * ns,), float("nan"), dtype=torch.float64, device=g.device)
    dt = nat.HIT_DTYPE_F32 if g.dtype == torch.float32 else nat.HIT_DTYPE_F64
    nat.call("hit_energy_spectrum_noalloc", g.Nx, g.Ny, g.Nz, g.Lx, g.Ly, g.Lz, dt, nat.ptr(u),
             nat.ptr(E), nat.ptr(Ec), nat.stream_ptr(g.device))
    return E.cpu().numpy(), Ec.view(3, ns).cpu().numpy()


TWO_PI = 2 * np.pi


# the last case is an anisotropic box (Ly = pi, Lz = 4 pi): the shell width
# comes from Lx, ky and kz are scaled by their own lengths, and shells past
# smax are dropped
@pytest.mark.parametrize("dims,dtype,lengths", [((64, 64, 64), torch.float32, (TWO_PI,) * 3),
                                                ((32, 16, 64), torch.float64, (TWO_PI,) * 3),
                                                ((64, 32, 16), torch.float32, (TWO_PI, np.pi, 2 * TWO_PI))])
def test_noalloc_spectrum_matches_plan_entry_point(h3, dims, dtype, lengths):
    nat = importlib.import_module("3dhit_b200._native")
    Lx, Ly, Lz = lengths
    g = h3.make_grid(*dims, Lx=Lx, Ly=Ly, Lz=Lz, dtype=dtype)
    fields = [h3.random_field(3, g), h3.hit_initial_field(4, g) * 0.5]
    for u in fields:  # two calls in a row on the shared scratch
        E, Ec = _noalloc(nat, g, u)
        _, E_ref = h3.energy_spectrum(u, g)
        _, c1, c2, c3 = h3.component_spectra(u, g)
        np.testing.assert_allclose(E, E_ref, rtol=1e-11, atol=1e-300)
        np.testing.assert_allclose(Ec, np.stack([c1, c2, c3]), rtol=1e-11, atol=1e-300)


def test_noalloc_rejects_oversize_grid(h3):
    nat = importlib.import_module("3dhit_b200._native")
    lib = nat.load()
    u = torch.zeros(8, dtype=torch.complex64, device="cuda")
    E = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = lib.hit_energy_spectrum_noalloc(2048, 2048, 2048, 6.28, 6.28, 6.28, nat.HIT_DTYPE_F32,
                                         ctypes.c_void_p(u.data_ptr()), ctypes.c_void_p(E.data_ptr()), None,
                                         None)
    assert rc == nat.HIT_E_UNSUPPORTED
    assert b"[4, 1024]" in lib.hit_last_error_string()
