"""Grid and spectral operators (reference: src/hit3d/grid.py).

`Grid` keeps the reference's fields (Nx..Lz, kx, ky, kz, k2, inv_k2, dealias,
weights) with the same values, as device tensors built lazily on first
access; the kernels never read them (they recompute wavenumbers, masks and
weights from indices).  Each grid owns one native plan per device.

Arrays are torch tensors on a CUDA device; inputs are never modified and
every function returns a new tensor, as the reference's pure functions do.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _native as nat

__all__ = ["Grid", "make_grid", "spectral_shape", "ddx", "ddy", "ddz", "laplacian",
           "dealias", "project", "to_physical", "to_spectral"]

_REAL = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64}


def _torch_real(dtype):
    if isinstance(dtype, torch.dtype):
        if dtype not in (torch.float32, torch.float64):
            raise ValueError(f"grid dtype must be float32 or float64, got {dtype}")
        return dtype
    return _REAL[np.dtype(dtype)]


class Grid:
    """Parameters and spectral operators of an Nx x Ny x Nz periodic box
    (src/hit3d/grid.py:41-86).  The broadcast shapes of kx, ky, kz and the
    full-grid k2 / inv_k2 / dealias / weights match the reference."""

    def __init__(self, Nx, Ny, Nz, Lx, Ly, Lz, dtype, device):
        self.Nx, self.Ny, self.Nz = int(Nx), int(Ny), int(Nz)
        self.Lx, self.Ly, self.Lz = float(Lx), float(Ly), float(Lz)
        self.dtype = _torch_real(dtype)
        self.cdtype = torch.complex64 if self.dtype == torch.float32 else torch.complex128
        self.device = torch.device(device)
        self._plan = None
        self._arrays = None

    # -- native plan --------------------------------------------------------
    @property
    def plan(self):
        if self._plan is None:
            self._plan = nat.Plan(self.Nx, self.Ny, self.Nz, self.Lx, self.Ly, self.Lz,
                                  self.dtype == torch.float64, self.device)
        return self._plan

    @property
    def num_shells(self):
        """smax = ceil(sqrt(3) max(N)/2) + 1 (src/hit3d/diagnostics.py:80)."""
        return int(np.ceil(np.sqrt(3) * max(self.Nx, self.Ny, self.Nz) / 2)) + 1

    # -- reference arrays (lazy) ---------------------------------------------
    def _build_arrays(self):
        npdt = np.float32 if self.dtype == torch.float32 else np.float64
        nx = np.fft.fftfreq(self.Nx, 1 / self.Nx)
        ny = np.fft.fftfreq(self.Ny, 1 / self.Ny)
        nz = np.arange(self.Nz // 2 + 1, dtype=float)
        kx = (2 * np.pi / self.Lx * nx).astype(npdt).reshape(-1, 1, 1)
        ky = (2 * np.pi / self.Ly * ny).astype(npdt).reshape(1, -1, 1)
        kz = (2 * np.pi / self.Lz * nz).astype(npdt).reshape(1, 1, -1)
        k2 = kx**2 + ky**2 + kz**2
        with np.errstate(divide="ignore"):
            inv_k2 = np.where(k2 == 0, npdt(0), 1 / k2).astype(npdt)
        mask = ((np.abs(nx).reshape(-1, 1, 1) <= self.Nx // 3)
                & (np.abs(ny).reshape(1, -1, 1) <= self.Ny // 3)
                & (np.abs(nz).reshape(1, 1, -1) <= self.Nz // 3))
        mask[0, 0, 0] = False
        w = np.full(self.Nz // 2 + 1, 2, dtype=npdt)
        w[0] = 1
        if self.Nz % 2 == 0:
            w[-1] = 1
        dev = self.device
        self._arrays = {
            "kx": torch.from_numpy(kx).to(dev), "ky": torch.from_numpy(ky).to(dev),
            "kz": torch.from_numpy(kz).to(dev), "k2": torch.from_numpy(k2).to(dev),
            "inv_k2": torch.from_numpy(inv_k2).to(dev),
            "dealias": torch.from_numpy(mask).to(dev),
            "weights": torch.from_numpy(w.reshape(1, 1, -1)).to(dev),
        }

    def __getattr__(self, name):
        if name in ("kx", "ky", "kz", "k2", "inv_k2", "dealias", "weights"):
            if self.__dict__.get("_arrays") is None:
                self._build_arrays()
            return self._arrays[name]
        raise AttributeError(name)

    def __repr__(self):
        dt = "float32" if self.dtype == torch.float32 else "float64"
        return (f"Grid[{dt}]({self.Nx}x{self.Ny}x{self.Nz}, "
                f"L=({self.Lx:g}, {self.Ly:g}, {self.Lz:g}))")


def make_grid(Nx, Ny=None, Nz=None, *, Lx=2 * np.pi, Ly=2 * np.pi, Lz=2 * np.pi,
              dtype=torch.float32, device=None):
    """``make_grid`` (src/hit3d/grid.py:89-132).  ``device`` defaults to the
    current CUDA device."""
    Ny = Nx if Ny is None else Ny
    Nz = Nx if Nz is None else Nz
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() \
            else torch.device("cuda", 0)
    return Grid(Nx, Ny, Nz, Lx, Ly, Lz, dtype, device)


def spectral_shape(grid):
    """``(3, Nx, Ny, Nz//2+1)`` (src/hit3d/grid.py:135-137)."""
    return (3, grid.Nx, grid.Ny, grid.Nz // 2 + 1)


# ---------------------------------------------------------------------------
# argument checking
# ---------------------------------------------------------------------------

def as_device(x, grid, dtype):
    """Tensor on the grid's device in ``dtype``, contiguous (numpy accepted)."""
    if not isinstance(x, torch.Tensor):
        x = torch.from_numpy(np.asarray(x))
    if x.device != grid.device or x.dtype != dtype:
        x = x.to(device=grid.device, dtype=dtype)
    return x.contiguous()


def _check_state(u_hat, grid):
    u_hat = as_device(u_hat, grid, grid.cdtype)
    if tuple(u_hat.shape) != spectral_shape(grid):
        raise ValueError(f"expected spectral state {spectral_shape(grid)}, got {tuple(u_hat.shape)}")
    return u_hat


# ---------------------------------------------------------------------------
# spectral operators
# ---------------------------------------------------------------------------

def ddx(u_hat, grid):
    """``i kx u`` (src/hit3d/grid.py:146-148)."""
    return 1j * grid.kx * as_device(u_hat, grid, grid.cdtype)


def ddy(u_hat, grid):
    """src/hit3d/grid.py:151-153."""
    return 1j * grid.ky * as_device(u_hat, grid, grid.cdtype)


def ddz(u_hat, grid):
    """src/hit3d/grid.py:156-158."""
    return 1j * grid.kz * as_device(u_hat, grid, grid.cdtype)


def laplacian(u_hat, grid):
    """``-k^2 u`` (src/hit3d/grid.py:161-163)."""
    return -grid.k2 * as_device(u_hat, grid, grid.cdtype)


def _dealias_project(u_hat, grid, dd, pp):
    u_hat = _check_state(u_hat, grid)
    out = torch.empty_like(u_hat)
    nat.call("hit_dealias_project", grid.plan.handle, nat.ptr(u_hat), int(dd), int(pp),
             nat.ptr(out), nat.stream_ptr(grid.device))
    return out


def dealias(u_hat, grid):
    """Zero the modes outside the 2/3 mask and k = 0 (src/hit3d/grid.py:166-168)."""
    u = as_device(u_hat, grid, grid.cdtype)
    if tuple(u.shape) == spectral_shape(grid):
        return _dealias_project(u, grid, 1, 0)
    return u * grid.dealias


def project(u_hat, grid):
    """Divergence-free projection (src/hit3d/grid.py:171-178)."""
    return _dealias_project(u_hat, grid, 0, 1)


def dealias_project(u_hat, grid):
    """``project(dealias(u_hat))`` in one pass."""
    return _dealias_project(u_hat, grid, 1, 1)


def to_physical(u_hat, grid):
    """irfftn over the three spatial axes (src/hit3d/grid.py:181-183); any
    number of leading components."""
    u_hat = as_device(u_hat, grid, grid.cdtype)
    sp = (grid.Nx, grid.Ny, grid.Nz // 2 + 1)
    if tuple(u_hat.shape[-3:]) != sp:
        raise ValueError(f"trailing shape must be {sp}, got {tuple(u_hat.shape)}")
    lead = u_hat.shape[:-3]
    flat = u_hat.reshape(-1, *sp)
    out = torch.empty((flat.shape[0], grid.Nx, grid.Ny, grid.Nz), dtype=grid.dtype, device=grid.device)
    st = nat.stream_ptr(grid.device)
    for c0 in range(0, flat.shape[0], 6):
        nc = min(6, flat.shape[0] - c0)
        nat.call("hit_to_physical", grid.plan.handle, nat.ptr(flat[c0]), nc, nat.ptr(out[c0]), st)
    return out.reshape(*lead, grid.Nx, grid.Ny, grid.Nz)


def to_spectral(u, grid):
    """Unnormalised rfftn (src/hit3d/grid.py:186-188)."""
    u = as_device(u, grid, grid.dtype)
    ph = (grid.Nx, grid.Ny, grid.Nz)
    if tuple(u.shape[-3:]) != ph:
        raise ValueError(f"trailing shape must be {ph}, got {tuple(u.shape)}")
    lead = u.shape[:-3]
    flat = u.reshape(-1, *ph)
    out = torch.empty((flat.shape[0], grid.Nx, grid.Ny, grid.Nz // 2 + 1), dtype=grid.cdtype,
                      device=grid.device)
    st = nat.stream_ptr(grid.device)
    for c0 in range(0, flat.shape[0], 6):
        nc = min(6, flat.shape[0] - c0)
        nat.call("hit_to_spectral", grid.plan.handle, nat.ptr(flat[c0]), nc, nat.ptr(out[c0]), st)
    return out.reshape(*lead, grid.Nx, grid.Ny, grid.Nz // 2 + 1)
