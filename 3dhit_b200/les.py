"""Coarse LES with the learned subgrid-stress closure.

* ``box_filter``: sharp spectral filter of a fine state to the coarse grid's
  2/3 box (|n_i| <= Nc/3), with the (Nc/Nf)^3 rescale of the unnormalised
  transform, giving the coarse spectral state of the filtered field.
* ``velocity_gradients``: du_i/dx_j of a state at its grid points (9 fields,
  ``hit_velocity_gradients``), the closure's input.
* ``sgs_stress``: the exact SGS stress of a fine state on the coarse grid,
  tau_ij = F(u_i u_j) - F(u_i) F(u_j) (xx, yy, zz, xy, xz, yz), the training
  target.
* ``LESRHS``: the coarse RHS, the fused Navier-Stokes RHS plus
  project(dealias(-d_j tau_ij)) of the closure's stress (``hit_add_sgs_force``);
  without a closure it is the unmodelled coarse solver.
* ``FusedLESStep``: one LES step on the fused step kernels, the closure's
  force held over the step (``hit_rollout_forced``).
* ``make_dataset`` / ``train`` / ``run_les``: the closure experiment
  (filtered forced DNS -> training -> LES against filtered DNS spectra).

The reference has no LES; this is the learned part of the package, built on the
package's own solver and kernels.
"""

from __future__ import annotations

import time

import torch

from . import _native as nat
from .closure import ClosureMLP, ctypes_ref
from .diagnostics import energy, energy_budget, energy_spectrum
from .fields import cfl_dt, hit_initial_field
from .forcing import HoldEnergyForcing, LinearForcing, native_params
from .grid import _check_state, make_grid, to_physical, to_spectral
from .integrators import rk4_step, rollout
from .navierstokes import NSParams, make_ns_rhs

__all__ = ["box_filter", "velocity_gradients", "sgs_stress", "LESRHS", "FusedLESStep", "make_dataset", "train",
           "run_les", "spectrum_log_loss", "les_window_grad", "train_a_posteriori"]

_PAIRS = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))


def _box_index(Nf, Nc, kc, device):
    src = torch.cat([torch.arange(0, kc + 1), torch.arange(Nf - kc, Nf)]).to(device)
    dst = torch.cat([torch.arange(0, kc + 1), torch.arange(Nc - kc, Nc)]).to(device)
    return src, dst


def box_filter(f_hat, fine, coarse):
    """Coarse spectral fields (any number of leading components) of the fine
    spectral fields ``f_hat`` restricted to |n_i| <= Nc/3."""
    kc = min(coarse.Nx, coarse.Ny, coarse.Nz) // 3
    lead = f_hat.shape[:-3]
    out = torch.zeros(*lead, coarse.Nx, coarse.Ny, coarse.Nz // 2 + 1, dtype=f_hat.dtype, device=f_hat.device)
    sx, dx = _box_index(fine.Nx, coarse.Nx, kc, f_hat.device)
    sy, dy = _box_index(fine.Ny, coarse.Ny, kc, f_hat.device)
    scale = (coarse.Nx * coarse.Ny * coarse.Nz) / (fine.Nx * fine.Ny * fine.Nz)
    sub = f_hat[..., :, :, : kc + 1].index_select(-3, sx).index_select(-2, sy)
    tmp = torch.zeros(*lead, coarse.Nx, sub.shape[-2], kc + 1, dtype=f_hat.dtype, device=f_hat.device)
    tmp.index_copy_(-3, dx, sub)
    tmp2 = torch.zeros(*lead, coarse.Nx, coarse.Ny, kc + 1, dtype=f_hat.dtype, device=f_hat.device)
    tmp2.index_copy_(-2, dy, tmp)
    out[..., : kc + 1] = tmp2 * scale
    return out


def velocity_gradients(u_hat, grid):
    """du_i/dx_j (component 3i + j) at the grid points, shape (9, N^3)."""
    u_hat = _check_state(u_hat, grid)
    P = grid.Nx * grid.Ny * grid.Nz
    g = torch.empty(9, P, dtype=grid.dtype, device=grid.device)
    nat.call("hit_velocity_gradients", grid.plan.handle, nat.ptr(u_hat), nat.ptr(g), nat.stream_ptr(grid.device))
    return g


def sgs_stress(u_hat_fine, fine, coarse):
    """Exact SGS stress of the filter on the coarse grid, shape (6, Nc^3)."""
    u = to_physical(u_hat_fine, fine)
    prods = torch.stack([u[i] * u[j] for i, j in _PAIRS])
    del u
    fuu = to_physical(box_filter(to_spectral(prods, fine), fine, coarse), coarse)
    ub = to_physical(box_filter(u_hat_fine, fine, coarse), coarse)
    tau = torch.stack([fuu[c] - ub[i] * ub[j] for c, (i, j) in enumerate(_PAIRS)])
    return tau.reshape(6, -1)


class LESRHS:
    """Coarse RHS with an optional learned closure (``ClosureMLP``).  With
    ``freeze_every`` = k the SGS stress is evaluated at every k-th call (the
    first stage of an RK4 step when k = 4) and reused in between."""

    def __init__(self, grid, closure=None, freeze_every=1):
        self.grid = grid
        self.ns = make_ns_rhs(grid)
        self.closure = closure
        self.freeze_every = int(freeze_every)
        self._tau = None
        self._tau_hat = None
        self._calls = 0

    def __call__(self, u_hat, params, t):
        g = self.grid
        du = self.ns(u_hat, params, t, assume_dealiased=True)
        if self.closure is not None:
            if self._calls % self.freeze_every == 0:
                P = g.Nx * g.Ny * g.Nz
                grads = velocity_gradients(u_hat, g)
                if self._tau is None:
                    self._tau = torch.empty(6, P, dtype=g.dtype, device=g.device)
                self.closure.forward_fields(grads, self._tau)
                self._tau_hat = to_spectral(self._tau.reshape(6, g.Nx, g.Ny, g.Nz), g)
            self._calls += 1
            nat.call("hit_add_sgs_force", g.plan.handle, nat.ptr(self._tau_hat), nat.ptr(du),
                     nat.stream_ptr(g.device))
        return du


class FusedLESStep:
    """One coarse-LES RK4 step on the fused step kernels: the closure's force
    f = project(dealias(-i k_j tau_hat_ij)) (``hit_velocity_gradients``, the
    MLP, one r2c of the six stress fields, ``hit_add_sgs_force``), held over
    the four stages of one fused RK4 step (``hit_rollout_forced``).  Without a
    closure it is the fused step of the unmodelled coarse solver.

    ``lag=False``: f from the step's initial state (the scheme of `LESRHS` with
    ``freeze_every`` = 4).  ``lag=True``: f from the previous step's initial
    state (the first call uses its own), computed on a second stream and a
    second plan of the same grid concurrently with the current step; the SGS
    term, already held over the RK stages, is then lagged by one step (first
    order in dt like the freeze itself), and at small grids, where the step
    kernels leave most SMs idle, the closure's cost is hidden.  All buffers are
    allocated at construction, so a call can be captured into a CUDA graph
    after one warm-up call.

    ``fused=True`` (unlagged, float32, Nz in {32, 64, 128}): the closure runs
    inside the step's own passes (`hit_les_rollout`): the first stage's
    x-inverse also emits the nine velocity gradients, its z pass evaluates the
    MLP per grid point on the tensor cores beside u x w, and its x-forward
    epilogue adds the force and holds it over the remaining stages -- the
    same scheme as ``fused=False`` without the separate gradient, MLP,
    transform and force launches."""

    def __init__(self, grid, closure, params, dt, lag=False, mlp_ctas_per_sm=1, fused=False):
        self.grid, self.closure, self.params, self.dt, self.lag = grid, closure, params, float(dt), bool(lag)
        self.fused = bool(fused) and closure is not None
        if self.fused and self.lag:
            raise ValueError("the fused closure evaluates the force inside the step: no lag")
        # with the lag the MLP shares the GPU with the step: a lighter footprint
        # (fewer CTAs per SM) keeps the step's kernels from waiting for SM space
        self.mlp_ctas_per_sm = int(mlp_ctas_per_sm) if self.lag else 0
        self.ns = make_ns_rhs(grid)
        P = grid.Nx * grid.Ny * grid.Nz
        dev = grid.device
        self._grads = torch.empty(9, P, dtype=grid.dtype, device=dev)
        self._tau = torch.empty(6, P, dtype=grid.dtype, device=dev)
        shape = (3, grid.Nx, grid.Ny, grid.Nz // 2 + 1)
        self._f = torch.zeros(shape, dtype=grid.cdtype, device=dev)
        if self.lag:
            # the closure's transforms on their own plan: plans are not re-entrant
            self._cgrid = make_grid(grid.Nx, grid.Ny, grid.Nz, Lx=grid.Lx, Ly=grid.Ly, Lz=grid.Lz,
                                    dtype=grid.dtype, device=dev)
            # two force buffers that swap roles every call (the step reads one,
            # the closure writes the other): consecutive calls alternate, so a
            # caller capturing CUDA graphs captures two (`graph_count`)
            self._fb = [self._f, torch.zeros(shape, dtype=grid.cdtype, device=dev)]
            self._i = 0
            # lowest priority: the step's kernels, on the caller's stream, go first
            lo, _ = torch.cuda.Stream.priority_range()
            self._side = torch.cuda.Stream(device=dev, priority=lo)
            self._primed = False

    def force(self, u_hat, grid=None, out=None):
        """The closure's force on u_hat into ``out`` (default: the step's
        buffer, reused by the next call), with ``grid``'s plan."""
        g = grid or self.grid
        out = self._f if out is None else out
        st = nat.stream_ptr(g.device)
        nat.call("hit_velocity_gradients", g.plan.handle, nat.ptr(u_hat), nat.ptr(self._grads), st)
        self.closure.forward_fields(self._grads, self._tau, self.mlp_ctas_per_sm)
        tau_hat = to_spectral(self._tau.reshape(6, g.Nx, g.Ny, g.Nz), g)
        nat.call("hit_sgs_force", g.plan.handle, nat.ptr(tau_hat), nat.ptr(out), st)
        return out

    def __call__(self, u_hat, out=None):
        """The state after one step (into ``out`` when given)."""
        u_hat = _check_state(u_hat, self.grid)
        if self.closure is None:
            return rk4_step(self.ns, u_hat, self.params, self.dt, 0.0, assume_dealiased=True, out=out)
        if self.fused:
            g = self.grid
            if getattr(self.closure, "_physical", None) is None:
                self.closure.pack_physical()
            p = native_params(self.params.nu, self.params.forcing, nat.HIT_FLAG_ASSUME_DEALIASED)
            out = torch.empty_like(u_hat) if out is None else out
            nat.call("hit_les_rollout", g.plan.handle, nat.ptr(u_hat), p, ctypes_ref(self.closure._physical[0]),
                     self.dt, 1, nat.ptr(out), nat.ptr(self.closure._err), nat.stream_ptr(g.device))
            return out
        if not self.lag:
            f = self.force(u_hat)
            return rk4_step(self.ns, u_hat, self.params, self.dt, 0.0, assume_dealiased=True, f_ext=f, out=out)
        cur, nxt = self._fb[self._i], self._fb[1 - self._i]
        if not self._primed:
            self.force(u_hat, self._cgrid, cur)
            self._primed = True
        main = torch.cuda.current_stream(self.grid.device)
        self._side.wait_stream(main)
        with torch.cuda.stream(self._side):
            self.force(u_hat, self._cgrid, nxt)
        out = rk4_step(self.ns, u_hat, self.params, self.dt, 0.0, assume_dealiased=True, f_ext=cur, out=out)
        main.wait_stream(self._side)
        self._i = 1 - self._i
        return out

    @property
    def graph_count(self):
        """CUDA graphs a caller captures to replay this step (2 with the lag:
        consecutive calls swap the force buffers)."""
        return 2 if self.lag and self.closure is not None else 1


def _spectrum(u_hat, grid, kmax):
    _, E = energy_spectrum(u_hat, grid)
    return torch.as_tensor(E[:kmax], dtype=torch.float64)


def make_dataset(fine_n=256, coarse_n=64, nu=1.5e-3, E_target=1.5, spinup=2000, snapshots=200, every=50, seed=0,
                 device="cuda", log=None):
    """Hold-energy (Lundgren) forced DNS on fine_n^3, filtered to coarse_n^3:
    features (S, 9, Pc) velocity gradients of the filtered field, targets
    (S, 6, Pc) the SGS stress, the filtered spectra, the forcing coefficient
    and the DNS step time."""
    fine = make_grid(fine_n, device=device)
    coarse = make_grid(coarse_n, device=device)
    forcing = HoldEnergyForcing(E_target, nu)
    p = NSParams(nu=nu, forcing=forcing)
    rhs = make_ns_rhs(fine)
    u = hit_initial_field(seed, fine)
    dt = cfl_dt(u, fine, 0.5)
    t0 = time.perf_counter()
    u = rollout(rhs, u, p, dt, spinup, assume_dealiased=True)
    torch.cuda.synchronize()
    Pc = coarse.Nx * coarse.Ny * coarse.Nz
    X = torch.empty(snapshots, 9, Pc, device=device)
    Y = torch.empty(snapshots, 6, Pc, device=device)
    spectra, A, E_f, U = [], [], [], []
    u0_coarse = None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dns_ms = 0.0
    kc = coarse_n // 3
    for s in range(snapshots):
        e0.record()
        u = rollout(rhs, u, p, dt, every, assume_dealiased=True)
        e1.record()
        torch.cuda.synchronize()
        dns_ms += e0.elapsed_time(e1)
        ub = box_filter(u, fine, coarse)
        if u0_coarse is None:
            u0_coarse = ub.clone()
        U.append(ub)
        X[s] = velocity_gradients(ub, coarse)
        Y[s] = sgs_stress(u, fine, coarse)
        spectra.append(_spectrum(ub, coarse, kc))
        E_f.append(float(energy(ub, coarse)))
        b = energy_budget(u, fine, nu, forcing)
        A.append(float(b["eps"]) / (2.0 * float(b["E"])))  # hold-energy A = 2 nu Omega / 2E
        if log and s % 20 == 0:
            log(f"snapshot {s}: E={float(b['E']):.4f}")
    return dict(X=X, Y=Y, U=torch.stack(U), spectra=torch.stack(spectra), A=A, E_filtered=E_f, dt=dt, nu=nu,
                dns_ms_per_step=dns_ms / (snapshots * every),
                u0_coarse=u0_coarse, fine=fine, coarse=coarse, wall_s=time.perf_counter() - t0)


def sgs_transfer(grads, tau):
    """Mean SGS energy transfer -<tau_ij S_ij> (S the resolved strain rate)
    of gradient fields (..., 9, P) and stress fields (..., 6, P)."""
    g = grads
    S = [g[..., 0, :], g[..., 4, :], g[..., 8, :], 0.5 * (g[..., 1, :] + g[..., 3, :]),
         0.5 * (g[..., 2, :] + g[..., 6, :]), 0.5 * (g[..., 5, :] + g[..., 7, :])]
    w = (1.0, 1.0, 1.0, 2.0, 2.0, 2.0)
    return -float(sum(w[c] * (tau[..., c, :].double() * S[c].double()).mean() for c in range(6)))


def train(data, steps=400, batch_snapshots=16, lr=2e-3, seed=0, val_snapshots=20, log=None):
    """Fit the closure on (X, Y) with Adam on the tensor-core gradients; the
    last ``val_snapshots`` snapshots are held out.  The fitted stress is then
    rescaled so that its mean SGS energy transfer -<tau_ij S_ij> over the
    training snapshots equals the DNS's (an MSE fit shrinks the stress towards
    zero and under-dissipates in the LES).  Returns the model and the loss
    history (train, validation)."""
    X, Y = data["X"], data["Y"]
    S = X.shape[0]
    ntr = S - val_snapshots
    m = ClosureMLP(X.device, seed=seed)
    m.x_scale = X[:ntr].transpose(0, 1).reshape(9, -1).std(1)
    m.y_scale = Y[:ntr].transpose(0, 1).reshape(6, -1).std(1)
    for q in m.params:
        q.requires_grad_(True)
    opt = torch.optim.Adam(m.params, lr=lr)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, steps)
    g = torch.Generator(device="cpu").manual_seed(seed)
    hist = []
    xs, ys = m.x_scale.view(1, 9, 1), m.y_scale.view(1, 6, 1)

    def batch(idx):
        xb = (X[idx] / xs).permute(0, 2, 1).reshape(-1, 9).contiguous()
        yb = (Y[idx] / ys).permute(0, 2, 1).reshape(-1, 6).contiguous()
        return xb, yb

    val = batch(torch.arange(ntr, S, device=X.device))
    for it in range(steps):
        idx = torch.randperm(ntr, generator=g)[:batch_snapshots].to(X.device)
        xb, yb = batch(idx)
        loss = m.loss_and_grads(xb, yb)
        opt.step()
        sched.step()
        m.pack()
        if it % 50 == 0 or it == steps - 1:
            vy = m.raw_forward(val[0])
            vl = float(((vy - val[1]) ** 2).mean())
            hist.append((it, float(loss.item()), vl))
            if log:
                log(f"step {it}: train {hist[-1][1]:.4f} val {vl:.4f}")
    m.check_errors()
    # energy-transfer calibration on the training snapshots
    pi_true, pi_model = 0.0, 0.0
    m.sgs_scale = 1.0
    m.pack_physical()
    out = torch.empty_like(Y[0])
    for s in range(ntr):
        m.forward_fields(X[s], out)
        pi_true += sgs_transfer(X[s], Y[s])
        pi_model += sgs_transfer(X[s], out)
    m.sgs_scale = pi_true / pi_model if pi_model > 0 else 1.0
    m._physical = None
    hist.append(("energy_transfer_true_model_scale", pi_true / ntr, pi_model / ntr, m.sgs_scale))
    if log:
        log(f"SGS transfer: DNS {pi_true / ntr:.4g}, fit {pi_model / ntr:.4g}, scale {m.sgs_scale:.3f}")
    return m, hist


def run_les(data, closure, steps=5000, sample_every=50, discard=1000, graph=True, tau_relax=0.5, freeze_every=4,
            fused=True, lag=False, forcing=None, fused_closure=False):
    """Coarse LES from the first filtered snapshot's state with the DNS's
    Lundgren forcing holding the total energy of the filtered DNS field (its
    mean over the snapshots; relaxation time ``tau_relax``), the SGS stress
    evaluated once per RK4 step (``freeze_every`` = 4; `FusedLESStep` when
    ``fused``, else the composed `LESRHS` step; ``fused_closure``: the closure
    inside the step's passes, see `FusedLESStep`; ``lag``: the fused step's
    lagged closure; ``forcing`` replaces the hold-energy forcing); returns the time-averaged
    spectrum over the samples after ``discard`` steps, the step time and the
    energy history."""
    coarse = data["coarse"]
    kc = coarse.Nx // 3
    E_res = sum(data["E_filtered"]) / len(data["E_filtered"])
    p = NSParams(nu=data["nu"], forcing=forcing or HoldEnergyForcing(E_res, data["nu"], tau=tau_relax))
    u = data["u0_coarse"].clone()
    dt = data.get("dt_les") or cfl_dt(u, coarse, 0.5)
    if fused and freeze_every == 4:
        step = FusedLESStep(coarse, closure, p, dt, lag=lag, fused=fused_closure)
    else:
        rhs = LESRHS(coarse, closure, freeze_every=freeze_every)

        def step(x, out=None):
            return rk4_step(rhs, x, p, dt, 0.0, out=out)

    run = step
    if graph:
        # the graphs advance the state between two buffers (graph k reads
        # bufs[k] and writes bufs[1-k]; with one graph the result is copied
        # back); with the lagged closure the two graphs also swap its force
        # buffers
        bufs = [u.clone(), torch.empty_like(u)]
        for _ in range(4):  # from the initial state; an even count keeps the lag's buffer parity
            step(bufs[0], out=bufs[1])
        torch.cuda.synchronize()
        ngraph = getattr(step, "graph_count", 1)
        _, hi = torch.cuda.Stream.priority_range()
        cap = torch.cuda.Stream(priority=hi)  # with the lag, the step's kernels go first
        graphs = []
        for k in range(ngraph):
            gph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(gph, stream=cap):
                if ngraph == 2:
                    step(bufs[k], out=bufs[1 - k])
                else:
                    bufs[0].copy_(step(bufs[0], out=bufs[1]))
            graphs.append(gph)
        turn = [0]

        def run(x):
            k = turn[0]
            if x is not bufs[k]:
                bufs[k].copy_(x)
            graphs[k].replay()
            turn[0] = (k + 1) % ngraph
            return bufs[1 - k] if ngraph == 2 else bufs[0]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    spec, n, energies = torch.zeros(kc, dtype=torch.float64), 0, []
    for i in range(1, steps + 1):
        u = run(u)
        if i % sample_every == 0:
            s = _spectrum(u, coarse, kc)
            energies.append(float(s.sum()))
            if i > discard:
                spec += s
                n += 1
    torch.cuda.synchronize()
    # timing: a clean window of 200 steps
    e0.record()
    for _ in range(200):
        u = run(u)
    e1.record()
    torch.cuda.synchronize()
    nat.check_device("run_les")
    if closure is not None and hasattr(closure, "check_errors"):
        closure.check_errors()
    return dict(spectrum=spec / max(n, 1), ms_per_step=e0.elapsed_time(e1) / 200, dt=dt, energies=energies,
                finite=bool(torch.isfinite(u).all()))


# ---------------------------------------------------------------------------
# a-posteriori tuning of the closure through the discrete adjoint
# ---------------------------------------------------------------------------

def spectrum_log_loss(u_hat, grid, logT):
    """L = sum_s (log E_s(u) - logT_s)^2 over shells s = 1..len(logT) (E_s the
    shell energies of `energy_spectrum`) and its cotangent with respect to
    u_hat (dL/dRe + i dL/dIm of every stored entry):
    2 (log E_s - logT_s) / E_s * w / N^6 * u_hat on the modes of shell s."""
    S = logT.numel()
    k0 = 2 * torch.pi / grid.Lx
    shp = u_hat.shape[1:]
    shell = torch.floor(torch.sqrt(grid.k2) / k0 + 0.5).to(torch.int64).expand(shp).reshape(-1)
    w = grid.weights.to(torch.float64).expand(shp).reshape(-1)
    n2 = float(grid.Nx * grid.Ny * grid.Nz) ** 2
    a2 = (u_hat.abs() ** 2).sum(0).reshape(-1).to(torch.float64)
    E = torch.bincount(shell.clamp(max=S + 1), weights=w * a2, minlength=S + 2)[: S + 1] / (2 * n2)
    r = torch.log(E[1:]) - logT.to(E.device, torch.float64)
    coef = torch.zeros(S + 2, dtype=torch.float64, device=u_hat.device)
    coef[1 : S + 1] = 2 * r / E[1:]
    c = (coef[shell.clamp(max=S + 1)] * w / n2).reshape(shp)
    return float((r ** 2).sum()), (c.to(u_hat.real.dtype) * u_hat).contiguous()


def les_window_grad(step, u0, nsteps, loss_fn):
    """Reverse-mode gradient of ``loss_fn(u_n)`` (returning the loss and its
    cotangent) after ``nsteps`` LES steps of `FusedLESStep` ``step`` (lag off)
    from u0, with respect to the closure's master parameters and to u0.

    The forward keeps every state (the coarse states are small); the backward
    runs, step by step from the last, the hand-written transposes:
    the RK4 step with its held force (``hit_rk4_step_forced_vjp``: the state's
    and the force's cotangents), the force f = P(-1j k_j rfftn(tau)_ij)
    (``hit_sgs_force_vjp``), the MLP (``hit_mlp_vjp``: parameter and input
    cotangents) and the velocity gradients (``hit_velocity_gradients_vjp``),
    the last two adding the closure's path to the state's cotangent.
    Returns (loss, parameter cotangents in the order of ``closure.params``,
    cotangent of u0, final state)."""
    from .forcing import native_params
    g = step.grid
    model = step.closure
    if model is None or step.lag:
        raise ValueError("les_window_grad needs a closure and lag=False")
    states = [_check_state(u0, g)]
    for _ in range(int(nsteps)):
        states.append(step(states[-1]))
    L, lam = loss_fn(states[-1])
    prm = native_params(step.params.nu, step.params.forcing, 0)
    if prm is None:
        raise ValueError("les_window_grad needs a built-in forcing")
    P = g.Nx * g.Ny * g.Nz
    st = nat.stream_ptr(g.device)
    gsum = [torch.zeros_like(q) for q in model.params]
    tbar = torch.empty(6, P, dtype=g.dtype, device=g.device)
    fbar = torch.empty_like(lam)
    for i in range(len(states) - 2, -1, -1):
        u = states[i]
        f = step.force(u)  # recomputed; leaves the gradient fields in step._grads
        ub = torch.empty_like(u)
        nat.call("hit_rk4_step_forced_vjp", g.plan.handle, nat.ptr(u), prm, nat.ptr(f), float(step.dt), 0.0,
                 nat.ptr(lam), nat.ptr(ub), nat.ptr(fbar), None, st)
        nat.call("hit_sgs_force_vjp", g.plan.handle, nat.ptr(fbar), nat.ptr(tbar), st)
        xbar, gp = model.vjp(step._grads, tbar)
        nat.call("hit_velocity_gradients_vjp", g.plan.handle, nat.ptr(xbar.to(g.dtype).contiguous()), nat.ptr(ub), st)
        for acc, d in zip(gsum, gp):
            acc += d
        lam = ub
    model.check_errors()
    nat.check_device("les_window_grad")
    return L, gsum, lam, states[-1]


def train_a_posteriori(data, model, iters=40, window=64, lr=3e-4, clip=1.0, tau_relax=0.5, seed=0, log=None,
                       select_every=0, select_steps=2000, val_snapshots=1):
    """Fine-tune a closure through the LES itself: each iteration runs the LES
    for ``window`` steps from a filtered DNS snapshot (the hold-energy forcing
    of `run_les`) and takes an Adam step on the gradient of the squared
    log-error of the final LES spectrum (shells 1..k_c) against the
    time-averaged filtered DNS spectrum, from `les_window_grad`; gradients
    are clipped to global norm ``clip``.  Returns the loss history.

    Model selection (``select_every`` > 0): the short windows only
    approximate what matters, the spectrum of a long LES run, and the
    stochastic descent through a chaotic LES can leave weights that do well
    on windows and drift on long runs.  The last ``val_snapshots`` snapshots
    are then kept out of the windows; before the first iteration, every
    ``select_every`` iterations and after the last, an LES of
    ``select_steps`` steps from the last held-out snapshot (time step from
    that snapshot's CFL condition, as `run_les` forms it) is scored by its
    maximum relative E(k) error (k <= k_c, samples after the first fifth)
    against the time-averaged filtered DNS spectrum, and the weights with the
    lowest score are restored at the end (the a-priori weights included).
    The scores are left in ``model.a_posteriori_selection`` as (iteration,
    score) pairs."""
    coarse = data["coarse"]
    kc = coarse.Nx // 3
    logT = torch.log(data["spectra"].mean(0)[:kc]).to(coarse.device)
    E_res = sum(data["E_filtered"]) / len(data["E_filtered"])
    p = NSParams(nu=data["nu"], forcing=HoldEnergyForcing(E_res, data["nu"], tau=tau_relax))
    U = data["U"]
    dt = data.get("dt_les") or cfl_dt(U[0], coarse, 0.5)
    for q in model.params:
        q.requires_grad_(False)
    opt = torch.optim.Adam(model.params, lr=lr)
    gen = torch.Generator().manual_seed(seed)
    hist = []
    ntrain = U.shape[0] - (val_snapshots if select_every > 0 else 0)
    if ntrain < 1:
        raise ValueError("no snapshots left for the windows after holding out the validation ones")
    sel, best = [], None
    ref = data["spectra"].mean(0)
    val_data = dict(data, u0_coarse=U[-1])

    def score(it):
        nonlocal best
        r = run_les(val_data, model, steps=select_steps, sample_every=50, discard=select_steps // 5,
                    tau_relax=tau_relax)
        sc = float((r["spectrum"] / ref - 1).abs().max()) if r["finite"] else float("inf")
        sel.append((it, sc))
        if best is None or sc < best[0]:
            best = (sc, [q.detach().clone() for q in model.params])
        if log:
            log(f"a-posteriori selection at {it}: max E(k) error {sc:.4f}")

    if select_every > 0:
        score(0)
    for it in range(iters):
        s = int(torch.randint(ntrain, (1,), generator=gen))
        step = FusedLESStep(coarse, model, p, dt)
        L, grads, _, _ = les_window_grad(step, U[s].clone(), window, lambda u: spectrum_log_loss(u, coarse, logT))
        norm = float(torch.sqrt(sum((d.double() ** 2).sum() for d in grads)))
        scale = min(1.0, clip / norm) if norm > 0 else 1.0
        for q, d in zip(model.params, grads):
            q.grad = d * scale
        opt.step()
        model._packed = None
        model._physical = None
        hist.append((it, s, L, norm))
        if log:
            log(f"a-posteriori {it}: snapshot {s}, loss {L:.4f}, |grad| {norm:.3g}")
        if select_every > 0 and ((it + 1) % select_every == 0 or it + 1 == iters):
            score(it + 1)
    if best is not None:
        with torch.no_grad():
            for q, b in zip(model.params, best[1]):
                q.copy_(b)
        model._packed = None
        model._physical = None
    model.a_posteriori_selection = sel
    return hist


def run_spectral_eddy_viscosity_les(data, steps, discard, coef=1.0, sample_every=50, tau_relax=0.5):
    """The coarse LES with the classical closure that needs no network: the
    Chollet-Lesieur spectral eddy viscosity
        nu_t(k) = coef C_K^(-3/2) (0.441 + 15.2 exp(-3.03 k_c / k)) sqrt(E(k_c) / k_c),
    C_K = 1.4 and E(k_c) the LES's own shell-k_c energy at the start of each
    step, applied as the force -nu_t(k) k^2 u_hat held over the step, under the
    hold-energy forcing of `run_les`.  Returns the spectrum of shells 1..k_c
    averaged over the samples taken every ``sample_every`` steps after
    ``discard``."""
    g, nu = data["coarse"], data["nu"]
    kc = g.Nx // 3
    E_res = sum(data["E_filtered"]) / len(data["E_filtered"])
    p = NSParams(nu=nu, forcing=HoldEnergyForcing(E_res, nu, tau=tau_relax))
    kmag = torch.sqrt(g.k2).clamp_min(1e-6)
    profile = (coef * 1.4 ** -1.5 * (0.441 + 15.2 * torch.exp(-3.03 * kc / kmag)) * g.k2).to(g.dtype)
    rhs = make_ns_rhs(g)
    u = data["u0_coarse"].clone()
    dt = data.get("dt_les") or cfl_dt(u, g, 0.5)
    total, count = torch.zeros(kc, dtype=torch.float64), 0
    for i in range(1, steps + 1):
        Ekc = max(float(energy_spectrum(u, g)[1][kc - 1]), 0.0)
        f = (-(Ekc / kc) ** 0.5 * profile) * u
        u = rk4_step(rhs, u, p, dt, 0.0, f_ext=f)
        if i % sample_every == 0 and i > discard:
            total += _spectrum(u, g, kc)
            count += 1
    return total / max(count, 1)
