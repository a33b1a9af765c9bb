"""Slab-decomposed RHS over several GPUs, one process per GPU.

The reference runs on one device (src/hit3d/navierstokes.py:62-97); this
module splits the same RHS over R ranks for grids that do not fit one GPU.

Layout.  Spectral arrays (components, Nx, Ny, Nz/2+1) are split along kx: rank
r holds kx rows [r Nx/R, (r+1) Nx/R) ("kx-slab").  Physical work arrays are
split along y ("y-slab": all x, y rows [r Ny/R, (r+1) Ny/R), all z).  One RHS:

  1. w_hat = 1j k x u_hat on the kx-slab (6 spectral fields with u_hat);
  2. inverse transform: along y (local to the kx-slab), all-to-all to the
     y-slab, along x, c2r along z (local to the y-slab) -- the axis order of
     irfftn (complex over x and y, then c2r over z, src/hit3d/grid.py:181-183);
  3. n = u x w on the y-slab;
  4. forward transform: r2c along z and forward along x (y-slab), all-to-all
     back to the kx-slab, forward along y;
  5. the epilogue on the kx-slab: forcing term (its sums over all modes
     all-reduced in float64), dealias mask, projection, -nu k^2 u_hat.

So an RHS moves 6 fields kx-slab -> y-slab and 3 back: two all-to-alls, each
rank sending (R-1)/R of its slab.  The exchanges are torch.distributed
all_to_all_single calls on device buffers (NCCL over NVLink on GPUs; nothing
here reads another GPU's memory directly, so no load of this path is a TMA or
bulk copy from peer memory).  The per-axis transforms are the package's CUDA
passes (``hit_axis_fft`` on plans of the slab shapes, `CudaSlabTransforms`);
the pointwise stages are device elementwise operations.  Any object with the
methods of `CudaSlabTransforms` can stand in for the transforms (the CPU
tests use one built on torch.fft).
"""

from __future__ import annotations

import math

import torch

from . import _native as nat
from .forcing import BandForcing, HoldEnergyForcing, LinearForcing, NoForcing

__all__ = ["SlabLayout", "to_y_slab", "to_kx_slab", "CudaSlabTransforms", "SlabRHS"]


class SlabLayout:
    """Rows of rank ``rank`` of ``world``: kx rows of the spectral slab, y rows
    of the physical slab (Nx and Ny divisible by world)."""

    def __init__(self, Nx, Ny, Nz, world, rank):
        if Nx % world or Ny % world:
            raise ValueError(f"Nx = {Nx} and Ny = {Ny} must be multiples of the {world} ranks")
        self.Nx, self.Ny, self.Nz, self.world, self.rank = Nx, Ny, Nz, world, rank
        self.nx = Nx // world
        self.ny = Ny // world
        self.Nzh = Nz // 2 + 1
        self.kx0 = rank * self.nx
        self.y0 = rank * self.ny

    def kx_rows(self):
        return slice(self.kx0, self.kx0 + self.nx)

    def y_rows(self):
        return slice(self.y0, self.y0 + self.ny)


def _exchange(send, group):
    recv = torch.empty_like(send)
    if group is None or torch.distributed.get_world_size(group) == 1:
        recv.copy_(send)
    else:
        torch.distributed.all_to_all_single(recv, send, group=group)
    return recv


def to_y_slab(a, lay, group=None):
    """(nc, Nx/R, Ny, Nzh) kx-slab -> (nc, Nx, Ny/R, Nzh) y-slab: chunk q of
    the y rows goes to rank q, and the received chunks stack along x in rank
    order."""
    nc, R = a.shape[0], lay.world
    send = a.reshape(nc, lay.nx, R, lay.ny, a.shape[-1]).permute(2, 0, 1, 3, 4).contiguous()
    recv = _exchange(send, group)  # [p] = rank p's kx rows of my y rows
    return recv.permute(1, 0, 2, 3, 4).reshape(nc, lay.Nx, lay.ny, a.shape[-1])


def to_kx_slab(b, lay, group=None):
    """(nc, Nx, Ny/R, Nzh) y-slab -> (nc, Nx/R, Ny, Nzh) kx-slab (the inverse
    of `to_y_slab`)."""
    nc, R = b.shape[0], lay.world
    send = b.reshape(nc, R, lay.nx, lay.ny, b.shape[-1]).permute(1, 0, 2, 3, 4).contiguous()
    recv = _exchange(send, group)  # [p] = my kx rows of rank p's y rows
    return recv.permute(1, 2, 0, 3, 4).reshape(nc, lay.nx, lay.Ny, b.shape[-1])


class CudaSlabTransforms:
    """Per-axis transforms of the slabs on the CUDA passes: a plan of the
    kx-slab's shape (Nx/R, Ny, Nz) for the y transforms and one of the
    y-slab's shape (Nx, Ny/R, Nz) for the x and z transforms (unnormalised,
    ``hit_axis_fft``)."""

    def __init__(self, lay, Lx, Ly, Lz, dtype, device):
        self.lay, self.device = lay, torch.device(device)
        f64 = dtype == torch.float64
        self.kx_plan = nat.Plan(lay.nx, lay.Ny, lay.Nz, Lx, Ly, Lz, f64, self.device)
        self.y_plan = nat.Plan(lay.Nx, lay.ny, lay.Nz, Lx, Ly, Lz, f64, self.device)

    def _call(self, plan, a, out, axis, inverse):
        nat.call("hit_axis_fft", plan.handle, nat.ptr(a), nat.ptr(out), a.shape[0], axis, int(inverse),
                 nat.stream_ptr(self.device))
        return out

    def y(self, a, inverse):  # kx-slab, complex along y
        return self._call(self.kx_plan, a.contiguous(), torch.empty_like(a), 1, inverse)

    def x(self, b, inverse):  # y-slab, complex along x
        return self._call(self.y_plan, b.contiguous(), torch.empty_like(b), 0, inverse)

    def z_c2r(self, b):  # y-slab, (nc, Nx, Ny/R, Nzh) complex -> (nc, Nx, Ny/R, Nz) real
        out = torch.empty(b.shape[0], self.lay.Nx, self.lay.ny, self.lay.Nz, dtype=b.real.dtype, device=b.device)
        return self._call(self.y_plan, b.contiguous(), out, 2, True)

    def z_r2c(self, r):  # y-slab real -> complex
        out = torch.empty(r.shape[0], self.lay.Nx, self.lay.ny, self.lay.Nzh, dtype=torch.complex64 if
                          r.dtype == torch.float32 else torch.complex128, device=r.device)
        return self._call(self.y_plan, r.contiguous(), out, 2, False)


class SlabRHS:
    """The RHS (src/hit3d/navierstokes.py:62-97) of this rank's kx-slab
    ``u_hat`` (3, Nx/R, Ny, Nz/2+1) of the global state: returns the rank's
    slab of du_hat.  ``params`` carries ``nu`` and a built-in forcing; the
    forcing's sums over all modes (band energy, E, Omega) are float64 partial
    sums all-reduced over ``group`` (None: one rank).  ``transforms``
    defaults to `CudaSlabTransforms`."""

    def __init__(self, Nx, Ny, Nz, Lx=2 * math.pi, Ly=2 * math.pi, Lz=2 * math.pi, dtype=torch.float32,
                 device=None, group=None, transforms=None):
        world = torch.distributed.get_world_size(group) if group is not None else 1
        rank = torch.distributed.get_rank(group) if group is not None else 0
        self.lay = lay = SlabLayout(Nx, Ny, Nz, world, rank)
        self.group = group
        self.dtype = dtype
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.T = transforms or CudaSlabTransforms(lay, Lx, Ly, Lz, dtype, self.device)

        def freqs(n, L):  # (T)(2 pi / L * n) from the float64 product, as make_grid
            f = torch.fft.fftfreq(n, 1.0 / n, dtype=torch.float64)
            return (2 * math.pi / L * f).to(dtype)

        nxf = torch.fft.fftfreq(Nx, 1.0 / Nx, dtype=torch.float64)[lay.kx_rows()]
        nyf = torch.fft.fftfreq(Ny, 1.0 / Ny, dtype=torch.float64)
        nzf = torch.arange(lay.Nzh, dtype=torch.float64)
        dev = self.device
        self.kx = freqs(Nx, Lx)[lay.kx_rows()].reshape(-1, 1, 1).to(dev)
        self.ky = freqs(Ny, Ly).reshape(1, -1, 1).to(dev)
        self.kz = (2 * math.pi / Lz * nzf).to(dtype).reshape(1, 1, -1).to(dev)
        self.k2 = self.kx * self.kx + self.ky * self.ky + self.kz * self.kz
        self.inv_k2 = torch.where(self.k2 > 0, 1.0 / torch.where(self.k2 > 0, self.k2, 1), 0).to(dtype)
        self.mask = ((nxf.abs() <= Nx // 3).reshape(-1, 1, 1) & (nyf.abs() <= Ny // 3).reshape(1, -1, 1)
                     & (nzf <= Nz // 3).reshape(1, 1, -1)).to(dev)
        if lay.kx0 == 0:
            self.mask[0, 0, 0] = False
        wz = torch.full((lay.Nzh,), 2.0, dtype=torch.float64)
        wz[0] = 1.0
        if Nz % 2 == 0:
            wz[-1] = 1.0
        self.w = wz.reshape(1, 1, -1).to(dev)
        self.ntot = float(Nx * Ny * Nz)

    def _allsum(self, v):
        t = torch.stack([torch.as_tensor(x, dtype=torch.float64, device=self.device) for x in v])
        if self.group is not None and self.lay.world > 1:
            torch.distributed.all_reduce(t, group=self.group)
        return t.tolist()

    def _forcing_term(self, u, forcing, nu):
        if isinstance(forcing, NoForcing) or forcing is None:
            return None
        if isinstance(forcing, LinearForcing):
            return float(forcing.A) * u
        a2 = (u.real.double() ** 2 + u.imag.double() ** 2).sum(0)
        n2 = self.ntot ** 2
        if isinstance(forcing, BandForcing):
            band = (float(forcing.kmin) ** 2 <= self.k2) & (self.k2 <= float(forcing.kmax) ** 2)
            two_eb = self._allsum([(self.w * band * a2).sum()])[0] / n2
            tiny = float(torch.finfo(self.dtype).eps)
            c = float(forcing.eps) / two_eb if two_eb > tiny else 0.0
            return (c * band.to(u.real.dtype)) * u
        if isinstance(forcing, HoldEnergyForcing):
            E, Om = self._allsum([(self.w * a2).sum(), (self.w * self.k2.double() * a2).sum()])
            E, Om = 0.5 * E / n2, 0.5 * Om / n2
            relax = 0.0 if not math.isfinite(forcing.tau) else (E - forcing.E_target) / forcing.tau
            A = (2.0 * float(forcing.nu) * Om - relax) / (2.0 * E) if E > 0 else 0.0
            return A * u
        raise TypeError(f"slab RHS: unsupported forcing {forcing!r}")

    def __call__(self, u_hat, params, t=0.0):
        lay, T = self.lay, self.T
        u = u_hat
        kx, ky, kz = self.kx, self.ky, self.kz
        w = 1j * torch.stack((ky * u[2] - kz * u[1], kz * u[0] - kx * u[2], kx * u[1] - ky * u[0]))
        f6 = torch.cat((u, w))
        # inverse: y (kx-slab) -> exchange -> x -> c2r along z (y-slab)
        phys = T.z_c2r(T.x(to_y_slab(T.y(f6, True), lay, self.group), True))
        s = 1.0 / self.ntot
        uu, ww = phys[:3], phys[3:]
        n = torch.stack((uu[1] * ww[2] - uu[2] * ww[1], uu[2] * ww[0] - uu[0] * ww[2],
                         uu[0] * ww[1] - uu[1] * ww[0])) * (s * s)
        # forward: r2c along z -> x (y-slab) -> exchange -> y (kx-slab)
        du = T.y(to_kx_slab(T.x(T.z_r2c(n), False), lay, self.group), False)
        ft = self._forcing_term(u, params.forcing, params.nu)
        if ft is not None:
            du = du + ft
        du = du * self.mask
        div = (kx * du[0] + ky * du[1] + kz * du[2]) * self.inv_k2
        du = du - torch.stack((kx * div, ky * div, kz * div))
        return du - float(params.nu) * self.k2 * u
