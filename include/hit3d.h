/*
 * hit3d.h -- C ABI of the B200-native HIT3D pseudo-spectral Navier-Stokes
 * hot path (sm_100a kernels in 3dhit_b200/csrc).
 *
 * Every entry point replaces one pure function of the reference JAX package
 * (nfrank22-gh/3DHIT, src/hit3d).  The spectral state is the reference's
 * layout: one complex array (ncomp, Nx, Ny, Nz/2+1), C order, components
 * first, rfft-halved axis last (src/hit3d/grid.py:7-14).  complex64 for
 * HIT_DTYPE_F32, complex128 for HIT_DTYPE_F64; physical fields are real
 * (ncomp, Nx, Ny, Nz).
 *
 * Conventions
 *  - All array arguments are DEVICE pointers owned by the caller; inputs are
 *    never modified (the reference functions are pure).  Output buffers may
 *    not alias inputs.
 *  - `stream` is a cudaStream_t passed as void*; every call is asynchronous
 *    on it.  A plan is bound to one stream at a time and is not re-entrant;
 *    separate plans are independent.
 *  - Workspace belongs to the plan.  It is allocated on first use of a
 *    code path (dealiased or general, see HIT_FLAG_ASSUME_DEALIASED) and then
 *    reused, so steady-state calls allocate nothing.
 *  - Return value: HIT_OK or a negative HIT_E* status; hit_last_error_string
 *    gives the message of the last failure on the calling thread.
 *  - Sizes: every N_i a power of two, 4 <= N_i <= 1024.
 */
#ifndef HIT3D_B200_H
#define HIT3D_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HIT_OK 0
#define HIT_E_INVALID (-1)     /* bad argument (shape, pointer, kind)        */
#define HIT_E_CUDA (-2)        /* a CUDA runtime call failed                  */
#define HIT_E_ALLOC (-3)       /* device allocation failed                    */
#define HIT_E_NONFINITE (-4)   /* non-finite value met by a checked reduction */
#define HIT_E_UNSUPPORTED (-5) /* size or dtype outside the supported set     */

#define HIT_DTYPE_F32 0
#define HIT_DTYPE_F64 1

/* Forcing plug-ins (src/hit3d/forcing.py:55-163) plus the energy-holding
 * Lundgren variant, which has no reference counterpart. */
#define HIT_FORCING_NONE 0        /* NoForcing      forcing.py:55-71          */
#define HIT_FORCING_LINEAR 1      /* LinearForcing  forcing.py:74-106 (f=A u) */
#define HIT_FORCING_BAND 2        /* BandForcing    forcing.py:109-163        */
#define HIT_FORCING_HOLD_ENERGY 3 /* A = (2 nu Omega - (E-E_target)/tau)/(2E) */

/* Flags (hit_params.flags). */
#define HIT_FLAG_ASSUME_DEALIASED 1u /* input is zero outside the 2/3 box: the
                                        transforms skip those modes           */
/* hit_rk4_step / hit_rollout advance with the integrating-factor (Lawson) RK4
 * on the viscous operator -nu k^2 (linear_operator, navierstokes.py:100-103;
 * the scheme the reference lists as to do, integrators.py:15-16):
 *   E = exp(-nu k^2 dt/2), N = rhs without its -nu k^2 u term,
 *   u' = E^2 u + dt/6 (E^2 k1 + 2E k2 + 2E k3 + k4),
 *   k1 = N(u), k2 = N(E(u + dt/2 k1)), k3 = N(E u + dt/2 k2),
 *   k4 = N(E^2 u + dt E k3).
 * No reference counterpart.  hit_rhs ignores it; the transposes reject it. */
#define HIT_FLAG_INTEGRATING_FACTOR 2u

typedef struct hit_plan hit_plan;

/* Differentiable scalars of the RHS: NSParams (src/hit3d/navierstokes.py:40-59)
 * and the forcing coefficients that are pytree leaves in the reference. */
typedef struct hit_params {
  double nu;         /* kinematic viscosity                                  */
  int forcing_kind;  /* HIT_FORCING_*                                        */
  unsigned flags;    /* HIT_FLAG_*                                           */
  double A;          /* LINEAR: coefficient                                  */
  double eps;        /* BAND: injection rate                                 */
  double kmin, kmax; /* BAND: shell limits |k| in [kmin, kmax]               */
  double E_target;   /* HOLD_ENERGY: held kinetic energy                     */
  double tau;        /* HOLD_ENERGY: relaxation time (<=0 or inf: none)      */
} hit_params;

/* make_grid (src/hit3d/grid.py:89-132): plan for an Nx x Ny x Nz box of
 * lengths Lx, Ly, Lz in the given dtype on the current CUDA device. */
int hit_plan_create(int nx, int ny, int nz, double lx, double ly, double lz,
                    int dtype, hit_plan **out);
int hit_plan_destroy(hit_plan *plan);

/* Number of shells returned by the spectrum calls:
 * smax = ceil(sqrt(3) max(N)/2) + 1 (src/hit3d/diagnostics.py:76-82). */
int hit_plan_num_shells(const hit_plan *plan);

/* to_physical (src/hit3d/grid.py:181-183): irfftn of ncomp components,
 * (ncomp,Nx,Ny,Nz/2+1) complex -> (ncomp,Nx,Ny,Nz) real.  1 <= ncomp <= 6. */
int hit_to_physical(hit_plan *plan, const void *u_hat, int ncomp, void *u,
                    void *stream);

/* to_spectral (src/hit3d/grid.py:186-188): unnormalised rfftn. */
int hit_to_spectral(hit_plan *plan, const void *u, int ncomp, void *u_hat,
                    void *stream);

/* dealias then project (src/hit3d/grid.py:166-178); either step can be
 * switched off (do_dealias / do_project = 0).  3 components. */
int hit_dealias_project(hit_plan *plan, const void *u_hat, int do_dealias,
                        int do_project, void *out, void *stream);

/* Per-shell rescale used by random_field (src/hit3d/fields.py:51-68):
 * out = u_hat * c[shell(k)] for 3 components, shell(k) = floor(|k|/k0 + 0.5)
 * as in the reference; c_dev is a DEVICE double array of
 * hit_plan_num_shells()+1 factors indexed by shell 0..smax (larger shells
 * clamp to smax, like jnp indexing). */
int hit_shell_scale(hit_plan *plan, const void *u_hat, const double *c_dev,
                    void *out, void *stream);

/* Writes 1 to *flag_dev (a device int) if u_hat has a nonzero mode outside
 * the 2/3 box, else 0.  Used to choose HIT_FLAG_ASSUME_DEALIASED. */
int hit_check_dealiased(hit_plan *plan, const void *u_hat, int *flag_dev,
                        void *stream);

/* rhs(u_hat, params, t) of make_ns_rhs (src/hit3d/navierstokes.py:62-97). */
int hit_rhs(hit_plan *plan, const void *u_hat, const hit_params *params,
            double t, void *du_hat, void *stream);

/* *status = 1 if a bounded wait of a transform kernel (the TMA tile loads of
 * the y and x passes) gave up since the last call, else 0; clears it.
 * Synchronises with the device.  No reference counterpart. */
int hit_device_status(int *status);

/* Test hook: the number of polls the tile/row-group waits of the TMA-staged
 * transform passes make before giving up, on the current device (polls < 0
 * restores the default of 2^22).  With 0 every such wait gives up at once:
 * the CTA raises the flag hit_device_status reports, waits (with the default
 * limit) for its copies in flight and ends, leaving its tiles untransformed.
 * It lets a test exercise the give-up path without stalling the GPU.  No
 * reference counterpart. */
int hit_set_wait_limit(int polls);

/* rhs and rollout with an external force f_ext (reference layout, device),
 * held constant over the call: rhs = project(dealias(u x w + forcing + f_ext))
 * - nu k^2 u, the RHS of a coarse LES whose subgrid-stress divergence is
 * evaluated once per step (the learned closure).  No reference counterpart:
 * the reference's rhs (src/hit3d/navierstokes.py:62-97) has only the forcing
 * plug-in, whose term must be a function of u_hat. */
int hit_rhs_forced(hit_plan *plan, const void *u_hat, const hit_params *params,
                   const void *f_ext, double t, void *du_hat, void *stream);
int hit_rollout_forced(hit_plan *plan, const void *u_hat,
                       const hit_params *params, const void *f_ext, double dt,
                       int64_t nsteps, double t0, void *out, void *stream);

/* rk4_step (src/hit3d/integrators.py:32-38). */
int hit_rk4_step(hit_plan *plan, const void *u_hat, const hit_params *params,
                 double dt, double t, void *out, void *stream);

/* rollout (src/hit3d/integrators.py:41-53): nsteps RK4 steps as one launch of
 * a CUDA graph that loops over the steps on the device (a while conditional
 * node counting down a step count in device memory; one step is enqueued
 * directly); no host synchronisation inside.  When the stream is
 * being captured by the caller (cudaStreamIsCapturing), the step kernels are
 * enqueued themselves, so a rollout can be part of the caller's graph (the
 * plan's buffers must exist by then: call once before capturing). */
int hit_rollout(hit_plan *plan, const void *u_hat, const hit_params *params,
                double dt, int64_t nsteps, double t0, void *out, void *stream);

/* Discrete adjoint (vector-Jacobian products).  The reference obtains these
 * with jax.vjp of rhs / rk4_step / rollout (src/hit3d/navierstokes.py:62-97,
 * src/hit3d/integrators.py:32-53).  Cotangents are arrays in the state layout
 * holding dL/dRe + i dL/dIm of the stored entries (PyTorch's convention; a JAX
 * custom_vjp rule conjugates them on the way in and out).  param_ct_dev, when
 * not NULL, is a DEVICE double[3] that receives the cotangents of (nu, A, eps)
 * of `params` (A: linear forcing; eps: band forcing; for the hold-energy
 * forcing nu also enters its coefficient).  The transposes run on the general
 * (full-layout) path in the plan's dtype and recompute what they need:
 *   hit_rhs_vjp       u_bar = (d rhs/d u)^T ct at u_hat;
 *   hit_rk4_step_vjp  u_bar = (d rk4_step/d u)^T ct (stage inputs recomputed);
 *   hit_rollout_vjp   u0_bar = (d rollout/d u0)^T ct: states are kept every
 *                     checkpoint_every steps, each segment is recomputed and
 *                     transposed step by step (memory: nsteps/checkpoint_every
 *                     + checkpoint_every states).
 * u_bar may alias ct. */
int hit_rhs_vjp(hit_plan *plan, const void *u_hat, const hit_params *params,
                double t, const void *ct, void *u_bar, double *param_ct_dev,
                void *stream);
int hit_rk4_step_vjp(hit_plan *plan, const void *u_hat,
                     const hit_params *params, double dt, double t,
                     const void *ct, void *u_bar, double *param_ct_dev,
                     void *stream);
int hit_rollout_vjp(hit_plan *plan, const void *u0_hat,
                    const hit_params *params, double dt, int64_t nsteps,
                    double t0, int checkpoint_every, const void *ct,
                    void *u0_bar, double *param_ct_dev, void *stream);

/* Measurement hook (no reference counterpart): the same nsteps RK4 steps as
 * hit_rollout, launched one kernel at a time with a CUDA event pair around
 * every launch on `stream`.  Host arrays ms_out / launches_out of
 * HIT_NUM_KERNEL_CLASSES entries receive, per kernel class, the summed device
 * time in ms and the number of launches.  Classes: 0 x-inverse (P1),
 * 1 y-inverse, 2 z pass (c2r, u x w, r2c), 3 y-forward, 4 x-forward + RHS/RK4
 * epilogue (+ next stage's x-inverse), 5 forcing coefficient.  Synchronises
 * `stream` before returning. */
#define HIT_NUM_KERNEL_CLASSES 6
int hit_profile_rollout(hit_plan *plan, const void *u_hat,
                        const hit_params *params, double dt, int64_t nsteps,
                        void *out, double *ms_out, int *launches_out,
                        void *stream);

/* energy_spectrum / component_spectra (src/hit3d/diagnostics.py:94-114),
 * accumulated in float64 (Kahan-compensated across blocks).  E_dev and
 * Ecomp_dev are DEVICE double arrays of hit_plan_num_shells() and
 * 3*hit_plan_num_shells() entries (either may be NULL); entry s is shell s+1. */
int hit_energy_spectrum(hit_plan *plan, const void *u_hat, double *E_dev,
                        double *Ecomp_dev, void *stream);

/* energy_budget (src/hit3d/diagnostics.py:162-172) in float64:
 * out_dev[0] = E, [1] = eps = 2 nu Omega, [2] = P (forcing injection),
 * [3] = Omega.  out_dev is a DEVICE double[4]. */
int hit_energy_budget(hit_plan *plan, const void *u_hat,
                      const hit_params *params, double *out_dev, void *stream);

/* BF16 GEMM on the fifth-generation tensor cores (no reference counterpart;
 * the building block of the learned subgrid-stress closure):
 *   C[M][N] (float32, row-major, ldc) = A[M][K] * B[N][K]^T
 * with A, B bf16 row-major (lda, ldb in elements, multiples of 8, 16-byte
 * aligned rows), N in {16, 32, 64, 128}, K a positive multiple of 16.
 * err_dev (DEVICE int) is set to 1 if a tensor-core wait timed out. */
int hit_tc_gemm_bf16(const void *A, int lda, const void *B, int ldb, float *C,
                     int ldc, int M, int N, int K, int *err_dev, void *stream);

/* Learned subgrid-stress closure for the coarse LES (no reference
 * counterpart): pointwise MLP 9 -> 64 -> 64 -> 64 -> 6 with GELU, bf16 weights
 * and activations, float32 accumulation, on the tcgen05 tensor cores.  Input
 * per point: the 9 filtered velocity-gradient components du_i/dx_j (i-major);
 * output: the 6 SGS stress components (xx, yy, zz, xy, xz, yz).  Weights are
 * DEVICE bf16 row-major arrays: the forward operands W^T of layers 1-4
 * ([64][16] with the layer-1 bias in input column 15, [64][64], [64][64],
 * [16][64]) and, for training, W of layers 2-4 ([64][64], [64][64],
 * [64][16]); biases b2, b3 ([64]) and b4 ([16]) float32. */
typedef struct hit_mlp_weights {
  const void *w1t, *w2t, *w3t, *w4t;
  const void *w2, *w3, *w4;
  const float *b2, *b3, *b4;
} hit_mlp_weights;

/* y[P][6] = MLP(x[P][9]) (DEVICE float32 arrays). */
int hit_mlp_forward(const hit_mlp_weights *w, const float *x, int64_t P,
                    float *y, int *err_dev, void *stream);
/* The same with strided arrays: feature f of point p at x[f*x_sf + p*x_sp],
 * output c at y[c*y_sf + p*y_sp] (component-major fields: x_sf = P, x_sp = 1).
 * ctas_per_sm: 0 = as many CTAs as fit (fastest alone); k > 0 = at most k per
 * SM (a lighter footprint when other kernels run concurrently). */
int hit_mlp_forward_strided(const hit_mlp_weights *w, const float *x,
                            int64_t x_sf, int64_t x_sp, int64_t P, float *y,
                            int64_t y_sf, int64_t y_sp, int ctas_per_sm,
                            int *err_dev, void *stream);

/* LES with the closure (no reference counterpart), reference layout:
 * grads_out (DEVICE, 9 x Nx*Ny*Nz, the plan's dtype) receives du_i/dx_j
 * (component 3i + j) at the grid points of the state u_hat;
 * hit_add_sgs_force adds project(dealias(-1j k_j tau_hat_ij)) to du_hat, tau_hat
 * holding the 6 spectral components xx, yy, zz, xy, xz, yz; hit_sgs_force
 * writes it to f_hat instead (every mode: zero outside the 2/3 box). */
int hit_velocity_gradients(hit_plan *plan, const void *u_hat, void *grads_out,
                           void *stream);
int hit_add_sgs_force(hit_plan *plan, const void *tau_hat, void *du_hat,
                      void *stream);
int hit_sgs_force(hit_plan *plan, const void *tau_hat, void *f_hat,
                  void *stream);

/* Coarse-LES rollout with the closure fused into the solver's passes (no
 * reference counterpart; the step it replaces is the reference RHS,
 * src/hit3d/navierstokes.py:69-95, plus the SGS force).  Every RK4 step
 * evaluates the closure at its initial state inside its first stage: the
 * x-inverse also emits the nine velocity gradients, the z pass forms w from
 * them, u x w and the MLP's six stresses per grid point (w: the same weights
 * as hit_mlp_forward_strided, inputs the gradients in physical units), and
 * the x-forward epilogue adds f = project(dealias(-1j k_j tau_hat_ij)) and
 * holds it over stages 2-4 (the scheme of hit_velocity_gradients +
 * hit_mlp_forward_strided + rfftn + hit_sgs_force + hit_rollout_forced with
 * nsteps = 1).  float32 plans, HIT_FLAG_ASSUME_DEALIASED, RK4, Nx <= 256 and
 * Nz in {32, 64, 128}; *err_dev is set when an MMA wait gave up.  Same
 * capture and graph behaviour as hit_rollout. */
int hit_les_rollout(hit_plan *plan, const void *u_hat, const hit_params *params,
                    const hit_mlp_weights *w, double dt, int64_t nsteps,
                    void *out, int *err_dev, void *stream);

/* Bytes of DEVICE workspace hit_mlp_train_grads needs for P points. */
int64_t hit_mlp_workspace_bytes(int64_t P);

/* Gradients of the mean-squared loss mean((MLP(x) - tau)^2) over P points
 * (P a multiple of 16): dW1 [16][64] (row 15 = d b1), dW2 and dW3 [65][64]
 * and dW4 [65][16] (row 64 = d b), float32 DEVICE arrays in [in][out]
 * order; loss_dev (DEVICE double) receives the loss.  The weight gradients
 * are tensor-core GEMMs over the points (split K). */
int hit_mlp_train_grads(const hit_mlp_weights *w, const float *x,
                        const float *tau, int64_t P, void *workspace,
                        float *dW1, float *dW2, float *dW3, float *dW4,
                        double *loss_dev, int *err_dev, void *stream);

/* One axis of the 3-D transform, unnormalised, on reference-layout arrays of
 * the plan's grid: axis 0 / 1 the complex transform along x / y of
 * (ncomp, Nx, Ny, Nz/2+1) complex arrays (in != out); axis 2 the real
 * transform along z between (ncomp, Nx, Ny, Nz/2+1) complex and
 * (ncomp, Nx, Ny, Nz) real (inverse = c2r, dropping the imaginary parts of
 * the kz = 0 and Nyquist entries as irfftn does; else r2c).  inverse != 0
 * selects exp(+2 pi i nk/N).  The building block of the slab-decomposed RHS
 * (3dhit_b200/slab.py): to_physical = z c2r after the x and y inverses
 * (src/hit3d/grid.py:181-183), each rank transforming its slab. */
int hit_axis_fft(hit_plan *plan, const void *in, void *out, int ncomp,
                 int axis, int inverse, void *stream);

/* Discrete adjoint of the coarse LES step with the learned closure (no
 * reference counterpart: the reference has no LES; its AD model is jax.vjp
 * through rollout, src/hit3d/integrators.py:5-9,41-53).  Cotangents follow
 * hit_rhs_vjp (dL/dRe + i dL/dIm of every stored entry).
 *
 * hit_rk4_step_forced_vjp: transpose of hit_rollout_forced(..., nsteps = 1),
 * the RK4 step with the force f_ext held over its stages: u_bar = (d step /
 * d u)^T ct, f_bar (nullable) = (d step / d f_ext)^T ct = P (sum of the
 * stages' cotangents), P the dealias mask and projection; param_ct as in
 * hit_rk4_step_vjp.  The stage inputs are recomputed on the general path. */
int hit_rk4_step_forced_vjp(hit_plan *plan, const void *u_hat,
                            const hit_params *params, const void *f_ext,
                            double dt, double t, const void *ct, void *u_bar,
                            void *f_bar, double *param_ct, void *stream);
/* tau_bar (DEVICE, 6 x Nx*Ny*Nz physical, the plan's dtype): the cotangent of
 * the physical stress tau whose force hit_sgs_force(rfftn(tau)) has cotangent
 * f_bar (reference layout). */
int hit_sgs_force_vjp(hit_plan *plan, const void *f_bar, void *tau_bar,
                      void *stream);
/* u_bar (reference layout) += the cotangent of u_hat whose velocity gradients
 * (hit_velocity_gradients) have cotangent grads_bar (9 x Nx*Ny*Nz physical). */
int hit_velocity_gradients_vjp(hit_plan *plan, const void *grads_bar,
                               void *u_bar, void *stream);
/* Vector-Jacobian product of the closure MLP at inputs x (feature f of point
 * p at x[f*x_sf + p*x_sp]) for the output cotangent ybar (component c at
 * ybar[c*y_sf + p*y_sp]): the parameter cotangents dW1..dW4 in the layout of
 * hit_mlp_train_grads, and, when xbar is not NULL, the input cotangent (same
 * layout as x); w1 is W1 as a bf16 [16][64] array (rows 0-8 used, the rest
 * zero), needed only for xbar.  P a multiple of 16; workspace of
 * hit_mlp_workspace_bytes(P) bytes. */
int hit_mlp_vjp(const hit_mlp_weights *w, const void *w1, const float *x,
                int64_t x_sf, int64_t x_sp, const float *ybar, int64_t y_sf,
                int64_t y_sp, int64_t P, void *workspace, float *dW1,
                float *dW2, float *dW3, float *dW4, float *xbar, int *err_dev,
                void *stream);

/* energy_spectrum without any device allocation.  No counterpart in the
 * reference: it serves callers that cannot allocate device memory -- code
 * running while its stream is being captured into a CUDA graph, an XLA custom
 * call that must take every buffer from XLA, a process whose device memory is
 * already reserved by another allocator.  Same outputs as hit_energy_spectrum
 * (E_dev: smax doubles, Ecomp_dev: 3*smax doubles, device pointers, either may
 * be NULL) for a grid given by its sizes, lengths and dtype; no plan is needed.
 * The per-block partial sums live in a fixed 4 MiB static device array held by
 * every GPU that loads this library until exit.  The first call on a device
 * (with that device current) looks up that array's address; make it before
 * any stream capture.  All calls share the array: calls that overlap on the
 * GPU race and must be ordered by the caller.  Grids are limited to powers of
 * two in [4, 1024] per axis; larger sizes are rejected with HIT_E_UNSUPPORTED. */
int hit_energy_spectrum_noalloc(int nx, int ny, int nz, double lx, double ly,
                                double lz, int dtype, const void *u_hat,
                                double *E_dev, double *Ecomp_dev, void *stream);

/* Message of the last failed call on this thread ("" if none). */
const char *hit_last_error_string(void);

#ifdef __cplusplus
}
#endif
#endif /* HIT3D_B200_H */
