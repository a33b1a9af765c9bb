"""Generate golden vectors by executing the reference's own source files.

jax/jaxlib cannot be installed in this environment (no network, no wheel), so
this script installs a minimal NumPy-backed stand-in for the handful of
``jax`` names the reference hot-path modules use (``jax.numpy`` array ops and
``numpy.fft`` transforms, identity ``jit``/``register_dataclass``, a Python
loop for ``lax.scan``) and then imports ``grid.py``, ``forcing.py``,
``navierstokes.py``, ``integrators.py`` and ``diagnostics.py`` unmodified from
the reference checkout.  Inputs come from the oracle's PCG64 ``random_field``
(``jax.random`` bits are not reproducible without jaxlib), so the same arrays
are fed to every implementation.  Outputs go to ``tests/golden/*.npz``.

Differences from a real jaxlib run, stated for the record: FFTs are
numpy.fft (pocketfft) instead of jaxlib's ducc0, float32 reductions are
NumPy's pairwise sums, and ``bincount`` accumulates in float64 before the cast
to the weights' dtype.

Usage (needs the reference checkout, so it runs only in the build container):
    python tests/golden/make_golden.py [/path/to/reference]
"""

from __future__ import annotations

import importlib
import os
import sys
import types
from functools import partial

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from oracle import hit3d_oracle as orc  # noqa: E402


def _install_jax_standin():
    jnp = types.ModuleType("jax.numpy")
    for name in ("asarray", "stack", "zeros", "sum", "abs", "finfo", "where",
                 "floor", "sqrt", "arange", "exp", "float32", "float64",
                 "complex64", "complex128", "int32", "promote_types", "ones",
                 "zeros_like", "real", "conj", "isfinite", "linalg"):
        setattr(jnp, name, getattr(np, name))
    jnp.fft = np.fft

    def bincount(x, weights=None, minlength=0, *, length=None):
        n = length if length is not None else max(minlength, int(x.max()) + 1)
        out = np.bincount(x, weights=weights, minlength=n)[:n]
        return out.astype(weights.dtype) if weights is not None else out

    jnp.bincount = bincount

    jax = types.ModuleType("jax")
    jax.numpy = jnp
    jax.Array = np.ndarray
    tu = types.ModuleType("jax.tree_util")
    tu.register_dataclass = lambda cls, data_fields=(), meta_fields=(): cls
    jax.tree_util = tu
    jax.jit = lambda f=None, **kw: (f if f is not None else (lambda g: g))
    lax = types.ModuleType("jax.lax")

    def scan(body, carry, xs):
        ys = []
        for x in xs:
            carry, y = body(carry, x)
            ys.append(y)
        return carry, ys

    lax.scan = scan
    jax.lax = lax
    jax.device_get = lambda x: x
    sys.modules.update({"jax": jax, "jax.numpy": jnp, "jax.tree_util": tu,
                        "jax.lax": lax, "h5py": types.ModuleType("h5py")})


def load_reference(ref_root):
    _install_jax_standin()
    src = os.path.join(ref_root, "src", "hit3d")
    pkg = types.ModuleType("hit3d")
    pkg.__path__ = [src]
    sys.modules["hit3d"] = pkg
    mods = {}
    for name in ("grid", "forcing", "navierstokes", "callbacks", "integrators",
                 "diagnostics"):
        mods[name] = importlib.import_module(f"hit3d.{name}")
    return types.SimpleNamespace(**mods)


def main(ref_root):
    ref = load_reference(ref_root)
    G, F, NS, I, D = ref.grid, ref.forcing, ref.navierstokes, ref.integrators, ref.diagnostics
    out = {}

    def forcings():
        return {"none": F.NoForcing(), "linear": F.LinearForcing(A=0.1333),
                "band": F.BandForcing(eps=0.1, kmin=1.0, kmax=2.0)}

    # --- grid arrays (float32/float64, cubic and anisotropic) -------------
    for tag, args, dt in (("g32f", (32,), np.float32), ("g16x8x4d", (16, 8, 4), np.float64),
                          ("g8f", (8,), np.float32)):
        g = G.make_grid(*args, dtype=dt)
        for fld in ("kx", "ky", "kz", "k2", "inv_k2", "dealias", "weights"):
            out[f"{tag}/{fld}"] = np.asarray(getattr(g, fld))

    # --- per-case vectors ---------------------------------------------------
    cases = [
        # tag, dims, dtype, seed, nu, dt
        ("c16f", (16, 16, 16), np.float32, 1, 0.02, 2e-3),
        ("c32f", (32, 32, 32), np.float32, 0, 0.02, 2e-3),
        ("c16x8x4d", (16, 8, 4), np.float64, 2, 0.05, 1e-3),
        ("c16d", (16, 16, 16), np.float64, 3, 0.02, 2e-3),
        ("a16x32x8f", (16, 32, 8), np.float32, 4, 0.02, 2e-3),
    ]
    for tag, dims, dt_, seed, nu, dt in cases:
        og = orc.make_grid(*dims, dtype=dt_)
        rg = G.make_grid(*dims, dtype=dt_)
        u0 = orc.hit_initial_field(seed, og, k0=2.0 if min(dims) < 16 else 4.0)
        out[f"{tag}/u0"] = u0
        out[f"{tag}/meta"] = np.array([nu, dt, seed], dtype=np.float64)
        out[f"{tag}/phys"] = np.asarray(G.to_physical(u0, rg))
        out[f"{tag}/spec_of_phys"] = np.asarray(G.to_spectral(out[f"{tag}/phys"], rg))
        rhs = NS.make_ns_rhs(rg)
        for fname, f in forcings().items():
            p = NS.NSParams(nu=nu, forcing=f)
            out[f"{tag}/rhs_{fname}"] = np.asarray(rhs(u0, p, 0.0))
            out[f"{tag}/step_{fname}"] = np.asarray(I.rk4_step(rhs, u0, p, dt, 0.0))
            b = D.energy_budget(u0, rg, nu, f)
            out[f"{tag}/budget_{fname}"] = np.array([float(b["E"]), float(b["eps"]), float(b["P"])])
        ks, Es = D.energy_spectrum(u0, rg)
        out[f"{tag}/spectrum"] = np.asarray(Es)
        out[f"{tag}/ks"] = np.asarray(ks)
        comp = D.component_spectra(u0, rg)
        out[f"{tag}/component_spectra"] = np.stack([np.asarray(c) for c in comp[1:]])
        out[f"{tag}/dealias_project"] = np.asarray(G.project(G.dealias(out[f"{tag}/spec_of_phys"], rg), rg))

    # --- config "plain decaying HIT 32^3": 100 RK4 steps, samples every 10 ---
    og = orc.make_grid(32, dtype=np.float32)
    rg = G.make_grid(32, dtype=np.float32)
    u = orc.hit_initial_field(0, og, k0=4.0)
    out["decay32/u0"] = u
    rhs = NS.make_ns_rhs(rg)
    p = NS.NSParams(nu=0.02)
    spectra, budgets = [], []
    for blk in range(10):
        ks, Es = D.energy_spectrum(u, rg)
        b = D.energy_budget(u, rg, 0.02, p.forcing)
        spectra.append(np.asarray(Es)); budgets.append([float(b["E"]), float(b["eps"]), float(b["P"])])
        u = np.asarray(I.rollout(rhs, u, p, 2e-3, 10, blk * 10 * 2e-3))
        if blk == 0:
            out["decay32/u10"] = u
    ks, Es = D.energy_spectrum(u, rg)
    b = D.energy_budget(u, rg, 0.02, p.forcing)
    spectra.append(np.asarray(Es)); budgets.append([float(b["E"]), float(b["eps"]), float(b["P"])])
    out["decay32/u100"] = u
    out["decay32/spectra"] = np.array(spectra)
    out["decay32/budgets"] = np.array(budgets)

    # --- Beltrami (float64, 32^3), reference conftest field ----------------
    g64 = G.make_grid(32, dtype=np.float64)
    ub = orc.beltrami(orc.make_grid(32, dtype=np.float64))
    out["beltrami/u0"] = ub
    out["beltrami/rhs"] = np.asarray(NS.make_ns_rhs(g64)(ub, NS.NSParams(nu=0.05), 0.0))

    path = os.path.join(HERE, "reference_vectors.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)/1e6:.2f} MB")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
