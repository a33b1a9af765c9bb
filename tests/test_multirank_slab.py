"""Slab-decomposed RHS (3dhit_b200/slab.py) as two and four gloo ranks on the CPU:
the kx-slab / y-slab partition and its all-to-all exchanges, with the local
per-axis transforms supplied here on torch.fft (the CUDA passes need a GPU),
against the oracle's RHS on the whole state in float64.  Unmeasured on GPU
hardware: this run has one GPU per call."""

import importlib
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import rel_l2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class TorchFFTSlabTransforms:
    """Unnormalised per-axis transforms of the slabs on torch.fft (CPU): the
    same contract as slab.CudaSlabTransforms."""

    def __init__(self, lay):
        self.lay = lay

    def y(self, a, inverse):
        return torch.fft.ifft(a, dim=2, norm="forward") if inverse else torch.fft.fft(a, dim=2)

    def x(self, b, inverse):
        return torch.fft.ifft(b, dim=1, norm="forward") if inverse else torch.fft.fft(b, dim=1)

    def z_c2r(self, b):  # irfft drops the imaginary parts of the kz = 0 and Nyquist entries, as irfftn does
        return torch.fft.irfft(b, n=self.lay.Nz, dim=3, norm="forward")

    def z_r2c(self, r):
        return torch.fft.rfft(r, dim=3)


def _forcings(slab):
    fm = importlib.import_module("3dhit_b200.forcing")
    return {"none": fm.NoForcing(), "linear": fm.LinearForcing(A=0.1333),
            "band": fm.BandForcing(eps=0.1, kmin=1.0, kmax=2.0), "hold": fm.HoldEnergyForcing(1.5, 0.02, tau=0.7)}


def _worker(rank, world, port, dims, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import hit3d_oracle as orc
        slab = importlib.import_module("3dhit_b200.slab")
        nav = importlib.import_module("3dhit_b200.navierstokes")
        og = orc.make_grid(*dims, dtype=np.float64)
        u = torch.as_tensor(orc.hit_initial_field(0, og, k0=2.0))
        lay = slab.SlabLayout(*dims, world, rank)
        # the exchanges invert each other
        a = u[:, lay.kx_rows()].contiguous()
        back = slab.to_kx_slab(slab.to_y_slab(a, lay, dist.group.WORLD), lay, dist.group.WORLD)
        res = {"roundtrip": bool(torch.equal(back, a))}
        rhs = slab.SlabRHS(*dims, dtype=torch.float64, device="cpu", group=dist.group.WORLD,
                           transforms=TorchFFTSlabTransforms(lay))
        for name, f in _forcings(slab).items():
            du = rhs(a, nav.NSParams(nu=0.02, forcing=f))
            res[name] = du.numpy()
        out[rank] = res
    finally:
        dist.destroy_process_group()


# four ranks exercise the all-to-all's block order, which two ranks cannot
# tell from its reverse
@pytest.mark.parametrize("world,dims", [(2, (16, 16, 16)), (2, (16, 8, 32)), (4, (16, 8, 32))])
def test_slab_rhs_matches_oracle(orc, world, dims):
    out = mp.Manager().dict()
    mp.start_processes(_worker, args=(world, _free_port(), dims, out), nprocs=world, start_method="spawn")
    og = orc.make_grid(*dims, dtype=np.float64)
    u = orc.hit_initial_field(0, og, k0=2.0)
    assert all(out[r]["roundtrip"] for r in range(world))
    forcings = {"none": orc.NoForcing(), "linear": orc.LinearForcing(A=0.1333),
                "band": orc.BandForcing(eps=0.1, kmin=1.0, kmax=2.0),
                "hold": orc.HoldEnergyForcing(1.5, 0.02, tau=0.7)}
    for name, f in forcings.items():
        ref = orc.make_ns_rhs(og)(u, orc.NSParams(nu=0.02, forcing=f), 0.0)
        got = np.concatenate([out[r][name] for r in range(world)], axis=1)  # kx slabs in rank order
        assert rel_l2(got, ref) < 1e-12, name
