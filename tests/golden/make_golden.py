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

A second file, ``tests/golden/reference_aux.npz``, holds what the
reference's driver-side code gives on the same inputs: the physical-space
diagnostics (``velocity_samples``, ``velocity_moments``,
``longitudinal_autocorrelation``, ``integral_lengthscale``), the steps at
which its ``Callback`` / ``Diagnostic`` / ``FieldWriter`` schedules fire, and
the steps at which ``evolve`` fires callbacks and prints progress.

Usage (needs the reference checkout; pass its root, or set HIT3D_REFERENCE):
    python tests/golden/make_golden.py /path/to/reference [--aux-only]
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


# schedule cases: (every_time, warmup_time, dt, t0, nsteps)
SCHEDULES = [
    (0.25, None, 1e-2, 0.0, 100), (0.5, 1.0, 0.1, 0.0, 30), (0.1, 0.0, 0.03, 0.0, 80),
    (0.07, 0.2, 0.013, 0.05, 150), (1.0 / 3.0, 0.5, 1.0 / 30.0, 0.0, 120), (0.2, 0.0, 0.05, 1.0, 60),
    (0.015, 0.0, 0.005, 0.0, 200), (0.3, 0.7, 0.1, 0.3, 40),
]


def aux(ref_root):
    """Physical-space diagnostics, callback schedules and evolve firing steps
    of the reference's own code (see the module docstring)."""
    import contextlib
    import io

    ref = load_reference(ref_root)
    G, NS, I, D, CB = ref.grid, ref.navierstokes, ref.integrators, ref.diagnostics, ref.callbacks
    out = {}
    for tag, dims, dt_, seed in (("c16f", (16, 16, 16), np.float32, 1), ("a16x32x8f", (16, 32, 8), np.float32, 4),
                                 ("c16d", (16, 16, 16), np.float64, 3)):
        og = orc.make_grid(*dims, dtype=dt_)
        rg = G.make_grid(*dims, dtype=dt_)
        u0 = orc.hit_initial_field(seed, og, k0=2.0 if min(dims) < 16 else 4.0)
        out[f"{tag}/u0"] = u0
        for c in range(3):
            smp = np.asarray(D.velocity_samples(u0, rg, component=c))
            out[f"{tag}/samples{c}"] = smp
            mom = D.velocity_moments(smp)
            out[f"{tag}/moments{c}"] = np.array([float(mom[k]) for k in ("mean", "variance", "skewness",
                                                                          "flatness")])
            r, f = D.longitudinal_autocorrelation(u0, rg, component=c)
            out[f"{tag}/autocorr_r{c}"] = np.asarray(r)
            out[f"{tag}/autocorr_f{c}"] = np.asarray(f)
            out[f"{tag}/lengthscale{c}"] = np.array([D.integral_lengthscale(r, f)])
    # schedules of the reference's wrappers
    for i, (every_time, warm, dt, t0, n) in enumerate(SCHEDULES):
        fw = CB.FieldWriter.__new__(CB.FieldWriter)  # is_due only: no file is made
        fw.every, fw.every_time = 1, every_time
        fw.warmup_time = 0.0 if warm is None else warm
        cb = CB.Callback(lambda s: None, every_time=every_time)
        out[f"sched{i}/case"] = np.array([every_time, -1.0 if warm is None else warm, dt, t0, n])
        out[f"sched{i}/fieldwriter"] = np.array([k for k in range(n + 1) if fw.is_due(k, t0 + k * dt, dt)])
        out[f"sched{i}/callback"] = np.array([k for k in range(n + 1) if cb.is_due(k, t0 + k * dt, dt)])
    # evolve: which steps fire which callback, and which steps print progress
    rg = G.make_grid(8, dtype=np.float64)
    u0 = orc.hit_initial_field(0, orc.make_grid(8, dtype=np.float64), k0=2.0)
    rhs = NS.make_ns_rhs(rg)
    for j, (nsteps, dt, every, every_time, progress) in enumerate(
            ((40, 0.03, 7, 0.25, 9), (25, 0.1, 4, 0.35, True), (13, 0.01, 5, None, False))):
        seen = {"cb": [], "diag": []}
        cbs = [CB.Callback(lambda s: seen["cb"].append(s.step), every_time=every_time) if every_time
               else CB.Callback(lambda s: seen["cb"].append(s.step), every=every),
               CB.Diagnostic(lambda s: (seen["diag"].append(s.step), 0.0)[1], every=every)]
        buf = io.StringIO()
        with contextlib.redirect_stdout(buf):
            I.evolve(rhs, u0, NS.NSParams(nu=0.05), rg, dt, nsteps, callbacks=cbs, progress=progress)
        printed = [int(line.split()[1].split("/")[0]) for line in buf.getvalue().splitlines() if line.strip()]
        out[f"evolve{j}/case"] = np.array([nsteps, dt, every, -1.0 if every_time is None else every_time,
                                           -1.0 if progress is True else float(progress)])
        out[f"evolve{j}/callback_steps"] = np.array(seen["cb"])
        out[f"evolve{j}/diagnostic_steps"] = np.array(seen["diag"])
        out[f"evolve{j}/progress_steps"] = np.array(printed)
    path = os.path.join(HERE, "reference_aux.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path)/1e6:.2f} MB")


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    root = args[0] if args else os.environ.get("HIT3D_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py /path/to/reference [--aux-only]  (or set HIT3D_REFERENCE)")
    if "--aux-only" not in sys.argv:
        main(root)
    aux(root)
