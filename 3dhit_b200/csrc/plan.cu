// Plan object and C ABI (include/hit3d.h).
//
// A plan is made per grid (make_grid, src/hit3d/grid.py:89-132).  It owns the
// wavenumber and twiddle tables and, per code path, the workspace of the
// fused RHS:
//   U, ACC, S, D  compact spectral state, RK accumulator, stage input, du
//   T6            x-physical u and w (6 comps); its first 3 comps later hold
//                 the y/z-forward products (T3)
//   U6            x,y-physical u and w (6 comps); first 3 comps: z-forward u x w
// One RHS evaluation (src/hit3d/navierstokes.py:69-95) is
//   P1 (x-inverse, k_p1)  -> P2a (y-inverse)  -> P2b (z c2r, u x w, z r2c)
//   -> P2c (y-forward)    -> P3 (x-forward + forcing/dealias/projection/
//                              viscous/RK update + next stage's P1)
// and one RK4 step (src/hit3d/integrators.py:32-38) is four such chains.  A
// rollout (integrators.py:41-53, the replacement for lax.scan) runs P1 once,
// then replays a captured CUDA graph of one step whose last P3 also prepares
// the next step's P1, and a final graph without that part.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <algorithm>

#include "fft_core.cuh"
#include "hit3d.h"
#include "kernels.h"

using namespace hit;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* where) {
  return fail(HIT_E_CUDA, std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

int ck(cudaError_t e, const char* where) { return e == cudaSuccess ? HIT_OK : cuda_fail(e, where); }

#define HIT_CK(expr)                                      \
  do {                                                    \
    cudaError_t _e = (expr);                              \
    if (_e != cudaSuccess) return cuda_fail(_e, #expr);   \
  } while (0)

struct Buf {
  void* p = nullptr;
  size_t bytes = 0;
};

int ensure(Buf& b, size_t bytes) {
  if (b.bytes >= bytes) return HIT_OK;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.bytes = 0;
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(HIT_E_ALLOC, "cudaMalloc(" + std::to_string(bytes) + " bytes) failed: " + cudaGetErrorString(e));
  }
  e = cudaMemset(b.p, 0, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemset(workspace)");
  b.bytes = bytes;
  return HIT_OK;
}
void release(Buf& b) {
  if (b.p) cudaFree(b.p);
  b = Buf{};
}

struct GraphKey {
  double nu, A, eps, kmin, kmax, E_target, tau, dt;
  int forcing, ifrk, fext;
  bool operator==(const GraphKey& o) const {
    return nu == o.nu && A == o.A && eps == o.eps && kmin == o.kmin && kmax == o.kmax && E_target == o.E_target &&
           tau == o.tau && dt == o.dt && forcing == o.forcing && ifrk == o.ifrk && fext == o.fext;
  }
};

struct Path {  // one code path: 0 = general (full layout), 1 = dealiased (2/3 box)
  Geom g{};
  bool ready = false;
  Buf t6, u6, U, ACC, S, D, partial, coef;
  Buf FEXT;  // external force held over a call (compact layout), see hit_rollout_forced
  int p3_blocks = 0, gather_blocks = 0;
  // the rollout graph: a device-side while loop over the steps that prepare
  // the next one, then the last step (see build_rollout_graph)
  cudaGraphExec_t exec = nullptr;
  Buf loop;  // int64 count of the loop's remaining steps
  GraphKey key{};
  // fused LES (hit_les_rollout): 12-field x- and y-pass buffers, its rollout
  // graph and the key it was built for (parameters and MLP weights)
  Buf t12, u12;
  cudaGraphExec_t les_exec = nullptr;
  GraphKey les_key{};
  hit_mlp_weights les_w{};
  int* les_err = nullptr;
  bool les_key_valid = false;
  bool key_valid = false;
};

Geom make_geom(int Nx, int Ny, int Nz, bool pruned) {
  Geom g{};
  g.Nx = Nx;
  g.Ny = Ny;
  g.Nz = Nz;
  g.H = Nz / 2;
  g.Nzh = Nz / 2 + 1;
  g.cx = Nx / 3;
  g.cy = Ny / 3;
  g.cz = Nz / 3;
  g.pruned = pruned ? 1 : 0;
  if (pruned) {
    g.Mx = 2 * g.cx + 1;
    g.hx = g.cx + 1;
    g.My = 2 * g.cy + 1;
    g.hy = g.cy + 1;
    g.Mz = g.cz + 1;
  } else {
    g.Mx = Nx;
    g.hx = Nx / 2;
    g.My = Ny;
    g.hy = Ny / 2;
    g.Mz = g.Nzh;
  }
  g.Mzp = (g.Mz + 7) / 8 * 8;
  return g;
}

bool pow2_ok(int n) { return n >= 4 && n <= 1024 && (n & (n - 1)) == 0; }

}  // namespace

struct hit_plan {
  int dtype = 0, Nx = 0, Ny = 0, Nz = 0;
  double Lx = 0, Ly = 0, Lz = 0;
  int device = 0;
  int smax = 0;
  Buf ktab, tw;
  Path path[2];
  Buf xws;                // to_physical / to_spectral workspace
  Buf dpartial, dsums;    // diagnostics partials / sums
  int diag_blocks = 0;
  // adjoint workspace (reference layout): transform inputs/outputs of the RHS
  // transpose, its float64 sums and scalars, the RK4 stage inputs and
  // cotangents, and the rollout checkpoints
  Buf ax9, aph, as6, apart, asums, ascal, apct, ast[3], ak, akb, asb, aacc, aub, ack, aseg, afb;
  cudaStream_t cap = nullptr;  // private stream used only for graph capture
  // side branch of the step for the forcing coefficient's reduction (see
  // fork_coef): its stream and one fork / join event pair per RK4 stage
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork[4] = {}, ev_join[4] = {};
};

namespace {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev);
    else prev = -1;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

template <typename T> KTab<T> ktab_of(const hit_plan* p) {
  const T* base = static_cast<const T*>(p->ktab.p);
  return KTab<T>{base, base + p->Nx, base + p->Nx + p->Ny};
}
template <typename T> const V2<T>* tw_of(const hit_plan* p) { return static_cast<const V2<T>*>(p->tw.p); }
template <typename T> V2<T>* vp(const Buf& b) { return static_cast<V2<T>*>(b.p); }

bool needs_coef(int forcing) { return forcing == HIT_FORCING_BAND || forcing == HIT_FORCING_HOLD_ENERGY; }

template <typename T> int ensure_path(hit_plan* p, int which) {
  Path& P = p->path[which];
  if (P.ready) return HIT_OK;
  P.g = make_geom(p->Nx, p->Ny, p->Nz, which == 1);
  const Geom& g = P.g;
  const size_t V = sizeof(V2<T>);
  const size_t cmp = (size_t)3 * g.Mx * g.My * g.Mzp * V;
  int rc;
  if ((rc = ensure(P.t6, (size_t)6 * g.Nx * g.My * g.Mzp * V))) return rc;
  if ((rc = ensure(P.u6, (size_t)6 * g.Nx * g.Ny * g.Mzp * V))) return rc;
  if ((rc = ensure(P.U, cmp))) return rc;
  if ((rc = ensure(P.ACC, cmp))) return rc;
  if ((rc = ensure(P.S, cmp))) return rc;
  if ((rc = ensure(P.D, cmp))) return rc;
  const int W = p3_tile_w<T>(g.Nx);
  P.p3_blocks = p3_num_blocks(g, W);
  const long long nm = (long long)g.Mx * g.My * g.Mzp;
  P.gather_blocks = (int)std::min<long long>((nm + NT - 1) / NT, 8 * 148);
  const int nb = std::max(P.p3_blocks, P.gather_blocks);
  if ((rc = ensure(P.partial, (size_t)3 * nb * sizeof(double)))) return rc;
  if ((rc = ensure(P.coef, 8 * sizeof(double)))) return rc;
  P.ready = true;
  return HIT_OK;
}

struct Scalars {
  int forcing;
  int ifrk;  // integrating-factor RK4 (HIT_FLAG_INTEGRATING_FACTOR)
  double nu, A, eps, kmin2, kmax2, E_target, tau;
};

Scalars scalars_of(const hit_params* pr) {
  Scalars s{};
  s.forcing = pr->forcing_kind;
  s.nu = pr->nu;
  s.A = pr->A;
  s.eps = pr->eps;
  s.kmin2 = pr->kmin * pr->kmin;
  s.kmax2 = pr->kmax * pr->kmax;
  s.E_target = pr->E_target;
  s.tau = pr->tau;
  s.ifrk = (pr->flags & HIT_FLAG_INTEGRATING_FACTOR) ? 1 : 0;
  return s;
}

// Optional per-launch event timer (hit_profile_rollout).
struct Prof {
  cudaStream_t st = nullptr;
  std::vector<cudaEvent_t> ev;
  std::vector<int> cls;
  int begin() { return mark(); }
  int end(int c) {
    cls.push_back(c);
    return mark();
  }
  int mark() {
    cudaEvent_t e;
    cudaError_t r = cudaEventCreate(&e);
    if (r != cudaSuccess) return cuda_fail(r, "cudaEventCreate");
    ev.push_back(e);
    r = cudaEventRecord(e, st);
    if (r != cudaSuccess) return cuda_fail(r, "cudaEventRecord");
    return HIT_OK;
  }
  ~Prof() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
  }
};

#define TIMED(pf, c, expr)                   \
  do {                                       \
    int _r;                                  \
    if ((pf) && (_r = (pf)->begin())) return _r; \
    if ((_r = (expr))) return _r;            \
    if ((pf) && (_r = (pf)->end(c))) return _r;  \
  } while (0)

template <typename T> double tiny_of() { return sizeof(T) == 4 ? (double)FLT_EPSILON : DBL_EPSILON; }
double ntot2_of(const hit_plan* p) {
  const double n = (double)p->Nx * p->Ny * p->Nz;
  return n * n;
}

template <typename T> int launch_coef(hit_plan* p, Path& P, const Scalars& s, int nblocks, cudaStream_t st) {
  CoefArgs c{};
  c.partial = static_cast<const double*>(P.partial.p);
  c.nblocks = nblocks;
  c.forcing = s.forcing;
  c.ntot2 = ntot2_of(p);
  c.nu = s.nu;
  c.eps = s.eps;
  c.E_target = s.E_target;
  c.tau = s.tau;
  c.tiny = tiny_of<T>();
  c.coef = static_cast<double*>(P.coef.p);
  HIT_CK(launch_finalize_coef(c, st));
  return HIT_OK;
}

// reference layout -> compact U (+ forcing coefficient of the gathered state)
template <typename T> int gather_state(hit_plan* p, Path& P, const void* u_hat, const Scalars& s, cudaStream_t st) {
  GatherArgs<T> a{};
  a.ext = static_cast<const V2<T>*>(u_hat);
  a.cmp = vp<T>(P.U);
  a.g = P.g;
  a.k = ktab_of<T>(p);
  a.kmin2 = (T)s.kmin2;
  a.kmax2 = (T)s.kmax2;
  a.partial = needs_coef(s.forcing) ? static_cast<double*>(P.partial.p) : nullptr;
  HIT_CK(launch_gather<T>(a, P.gather_blocks, st));
  if (needs_coef(s.forcing)) return launch_coef<T>(p, P, s, P.gather_blocks, st);
  return HIT_OK;
}

template <typename T> int launch_p1_of(hit_plan* p, Path& P, const V2<T>* src, cudaStream_t st, bool les = false) {
  const Geom& g = P.g;
  P1Args<T> a{};
  a.s = src;
  a.s_c = (long long)g.Mx * g.My * g.Mzp;
  a.s_x = (long long)g.My * g.Mzp;
  a.les = les ? 1 : 0;
  a.t6 = vp<T>(les ? P.t12 : P.t6);
  a.t_c = (long long)g.Nx * g.My * g.Mzp;
  a.t_x = (long long)g.My * g.Mzp;
  a.g = g;
  a.k = ktab_of<T>(p);
  a.tw = tw_of<T>(p);
  HIT_CK(launch_p1<T>(a, st));
  return HIT_OK;
}

// P2a, P2b, P2c: T6 -> U6 (y-inverse), z pass in place on U6, U6[0:3] -> T6[0:3]
template <typename T> int launch_p2(hit_plan* p, Path& P, cudaStream_t st, Prof* pf = nullptr) {
  const Geom& g = P.g;
  const long long t6c = (long long)g.Nx * g.My * g.Mzp, u6c = (long long)g.Nx * g.Ny * g.Mzp;
  const int Wy = axis_tile_w<T>(g.Ny);
  AxisArgs<T> a{};
  a.src = vp<T>(P.t6);
  a.dst = vp<T>(P.u6);
  a.s_c = t6c;
  a.s_a = g.Mzp;
  a.s_o = (long long)g.My * g.Mzp;
  a.d_c = u6c;
  a.d_a = g.Mzp;
  a.d_o = (long long)g.Ny * g.Mzp;
  a.Min = g.My;
  a.hin = g.hy;
  a.Mout = g.Ny;
  a.hout = g.Ny / 2;
  a.nz = g.Mzp;
  a.tw = tw_of<T>(p);
  TIMED(pf, 1, ck(launch_axis<T>(g.Ny, true, a, g.Mzp / Wy, g.Nx, 6, st), "y-inverse"));

  ZCrossArgs<T> z{};
  z.buf = vp<T>(P.u6);
  z.c_stride = u6c;
  z.nrows = g.Nx * g.Ny;
  z.Mz = g.Mz;
  z.Mzp = g.Mzp;
  z.scale = (T)(1.0 / ((double)g.Nx * g.Ny * g.Nz));
  z.tw = tw_of<T>(p);
  TIMED(pf, 2, ck(launch_zcross<T>(g.H, z, st), "z pass"));

  AxisArgs<T> b{};
  b.src = vp<T>(P.u6);
  b.dst = vp<T>(P.t6);
  b.s_c = u6c;
  b.s_a = g.Mzp;
  b.s_o = (long long)g.Ny * g.Mzp;
  b.d_c = t6c;
  b.d_a = g.Mzp;
  b.d_o = (long long)g.My * g.Mzp;
  b.Min = g.Ny;
  b.hin = g.Ny / 2;
  b.Mout = g.My;
  b.hout = g.hy;
  b.nz = g.Mzp;
  b.tw = tw_of<T>(p);
  TIMED(pf, 3, ck(launch_axis<T>(g.Ny, false, b, g.Mzp / Wy, g.Nx, 3, st), "y-forward"));
  return HIT_OK;
}

// P2 of the fused LES stage (float32): T12 -> U12 (y-inverse of u and the
// nine velocity gradients), the LES z pass in place on U12 (u x w, the
// closure MLP, r2c of the products and the stresses), U12[0:9] -> T12[0:9]
// (y-forward).
int launch_p2_les(hit_plan* p, Path& P, const hit_mlp_weights& w, int* err, cudaStream_t st) {
  const Geom& g = P.g;
  const long long tc = (long long)g.Nx * g.My * g.Mzp, uc = (long long)g.Nx * g.Ny * g.Mzp;
  const int Wy = axis_tile_w<float>(g.Ny);
  AxisArgs<float> a{};
  a.src = vp<float>(P.t12);
  a.dst = vp<float>(P.u12);
  a.s_c = tc;
  a.s_a = g.Mzp;
  a.s_o = (long long)g.My * g.Mzp;
  a.d_c = uc;
  a.d_a = g.Mzp;
  a.d_o = (long long)g.Ny * g.Mzp;
  a.Min = g.My;
  a.hin = g.hy;
  a.Mout = g.Ny;
  a.hout = g.Ny / 2;
  a.nz = g.Mzp;
  a.tw = tw_of<float>(p);
  HIT_CK(launch_axis<float>(g.Ny, true, a, g.Mzp / Wy, g.Nx, 12, st));
  ZLesArgs z{};
  z.buf = vp<float>(P.u12);
  z.c_stride = uc;
  z.nrows = g.Nx * g.Ny;
  z.Mz = g.Mz;
  z.Mzp = g.Mzp;
  z.scale = (float)(1.0 / ((double)g.Nx * g.Ny * g.Nz));
  z.tw = tw_of<float>(p);
  z.w1t = static_cast<const __nv_bfloat16*>(w.w1t);
  z.w2t = static_cast<const __nv_bfloat16*>(w.w2t);
  z.w3t = static_cast<const __nv_bfloat16*>(w.w3t);
  z.w4t = static_cast<const __nv_bfloat16*>(w.w4t);
  z.b2 = w.b2;
  z.b3 = w.b3;
  z.b4 = w.b4;
  z.err = err;
  HIT_CK(launch_zles(g.H, z, st));
  AxisArgs<float> b{};
  b.src = vp<float>(P.u12);
  b.dst = vp<float>(P.t12);
  b.s_c = uc;
  b.s_a = g.Mzp;
  b.s_o = (long long)g.Ny * g.Mzp;
  b.d_c = tc;
  b.d_a = g.Mzp;
  b.d_o = (long long)g.My * g.Mzp;
  b.Min = g.Ny;
  b.hin = g.Ny / 2;
  b.Mout = g.My;
  b.hout = g.hy;
  b.nz = g.Mzp;
  b.tw = tw_of<float>(p);
  HIT_CK(launch_axis<float>(g.Ny, false, b, g.Mzp / Wy, g.Nx, 9, st));
  return HIT_OK;
}

// les_in: the fused LES stage (x-forward of T12's nine fields, the force
// -i k_j tau_hat_ij added and stored in FEXT); les_next: the fused x-inverse
// is the LES one (12 fields into T12), for a following fused LES stage.
template <typename T>
int launch_p3_stage(hit_plan* p, Path& P, const Scalars& s, int stage, double dt, bool fuse, bool partial,
                    const V2<T>* fext, cudaStream_t st, bool les_in = false, bool les_next = false) {
  const Geom& g = P.g;
  P3Args<T> a{};
  a.t3 = vp<T>(les_in ? P.t12 : P.t6);
  a.les = les_in ? 1 : 0;
  a.fext_out = les_in ? vp<T>(P.FEXT) : nullptr;
  a.t_c = (long long)g.Nx * g.My * g.Mzp;
  a.t_x = (long long)g.My * g.Mzp;
  a.u = vp<T>(P.U);
  a.acc = vp<T>(P.ACC);
  a.s = vp<T>(P.S);
  a.out = vp<T>(P.D);
  a.c_c = (long long)g.Mx * g.My * g.Mzp;
  a.c_x = (long long)g.My * g.Mzp;
  a.t6 = vp<T>(fuse && les_next ? P.t12 : P.t6);
  a.t6_c = a.t_c;
  a.t6_x = a.t_x;
  a.g = g;
  a.k = ktab_of<T>(p);
  a.tw = tw_of<T>(p);
  a.stage = stage;
  a.fuse_p1 = fuse ? (les_next ? 2 : 1) : 0;
  a.ifrk = stage > 0 && s.ifrk ? 1 : 0;
  a.nu = a.ifrk ? (T)0 : (T)s.nu;
  a.nuh = (T)(0.5 * dt * s.nu);
  a.a_next = stage == 3 ? (T)dt : (T)(0.5 * dt);
  a.dt6 = (T)(dt / 6.0);
  a.forcing = s.forcing;
  a.fA = (T)s.A;
  a.kmin2 = (T)s.kmin2;
  a.kmax2 = (T)s.kmax2;
  a.coef = static_cast<const double*>(P.coef.p);
  a.partial = partial ? static_cast<double*>(P.partial.p) : nullptr;
  a.fext = fext;
  HIT_CK(launch_p3<T>(a, st));
  return HIT_OK;
}

// One RK4 step on the compact state U (P1 first, then four RHS chains).
// One RK4 step on the compact state U, starting from the x-inverse of U in T6
// (left by the previous step's last stage or by a standalone k_p1).  With
// fuse_next the last stage also runs the x-inverse of the new state for the
// following step.
// The forcing coefficient of the next stage input, reduced on a side branch
// of the step: fork after the k_p3 that wrote its partial sums, join just
// before the k_p3 that reads it, so that the one-block reduction runs beside
// the next stage's y-inverse, z pass and y-forward instead of between them
// (in a captured graph: a parallel branch with its own edges).
template <typename T> int fork_coef(hit_plan* p, Path& P, const Scalars& s, int k, cudaStream_t st) {
  HIT_CK(cudaEventRecord(p->ev_fork[k], st));
  HIT_CK(cudaStreamWaitEvent(p->side, p->ev_fork[k], 0));
  int rc;
  if ((rc = launch_coef<T>(p, P, s, P.p3_blocks, p->side))) return rc;
  HIT_CK(cudaEventRecord(p->ev_join[k], p->side));
  return HIT_OK;
}
int join_coef(hit_plan* p, int k, cudaStream_t st) {
  HIT_CK(cudaStreamWaitEvent(st, p->ev_join[k], 0));
  return HIT_OK;
}

template <typename T>
int enqueue_step(hit_plan* p, Path& P, const Scalars& s, double dt, bool fuse_next, const V2<T>* fext,
                 cudaStream_t st, Prof* pf = nullptr) {
  int rc;
  const bool red = needs_coef(s.forcing);
  const bool branch = red && !pf;  // timed runs keep every kernel on the one stream
  for (int stage = 1; stage <= 4; ++stage) {
    if ((rc = launch_p2<T>(p, P, st, pf))) return rc;
    if (branch && stage > 1 && (rc = join_coef(p, stage - 2, st))) return rc;
    TIMED(pf, 4, launch_p3_stage<T>(p, P, s, stage, dt, stage < 4 || fuse_next, red, fext, st));
    if (branch) {
      if ((rc = fork_coef<T>(p, P, s, stage - 1, st))) return rc;
    } else if (red) {
      TIMED(pf, 5, launch_coef<T>(p, P, s, P.p3_blocks, st));
    }
  }
  if (branch && (rc = join_coef(p, 3, st))) return rc;  // the next step's first stage reads it
  return HIT_OK;
}

// One RK4 step of the coarse LES with the learned closure fused into its
// first stage (float32, dealiased path): stage 1 runs the LES passes (the
// closure's force f = -i k_j tau_hat_ij from the step's initial state, added
// to that stage's nonlinear term and stored in FEXT), stages 2-4 the plain
// passes with f held (the scheme of hit_rollout_forced with the force of
// hit_sgs_force).  Starts from the LES x-inverse of U in T12; with fuse_next
// the last stage runs the next step's LES x-inverse.
int enqueue_les_step(hit_plan* p, Path& P, const Scalars& s, double dt, bool fuse_next, const hit_mlp_weights& w,
                     int* err, cudaStream_t st) {
  int rc;
  const bool red = needs_coef(s.forcing);
  const float2* f = vp<float>(P.FEXT);
  for (int stage = 1; stage <= 4; ++stage) {
    if (stage == 1) {
      if ((rc = launch_p2_les(p, P, w, err, st))) return rc;
      if ((rc = launch_p3_stage<float>(p, P, s, 1, dt, true, red, nullptr, st, true, false))) return rc;
    } else {
      if ((rc = launch_p2<float>(p, P, st))) return rc;
      if (red && (rc = join_coef(p, stage - 2, st))) return rc;
      if ((rc = launch_p3_stage<float>(p, P, s, stage, dt, stage < 4 || fuse_next, red, f, st, false,
                                       stage == 4 && fuse_next)))
        return rc;
    }
    if (red && (rc = fork_coef<float>(p, P, s, stage - 1, st))) return rc;
  }
  if (red && (rc = join_coef(p, 3, st))) return rc;
  return HIT_OK;
}

template <typename T>
int profile_impl(hit_plan* p, const void* u_hat, const hit_params* pr, double dt, int64_t nsteps, void* out,
                 double* ms, int* launches, cudaStream_t st) {
  int rc;
  const int which = (pr->flags & HIT_FLAG_ASSUME_DEALIASED) ? 1 : 0;
  if ((rc = ensure_path<T>(p, which))) return rc;
  Path& P = p->path[which];
  const Scalars s = scalars_of(pr);
  if ((rc = gather_state<T>(p, P, u_hat, s, st))) return rc;
  Prof pf;
  pf.st = st;
  TIMED(&pf, 0, launch_p1_of<T>(p, P, vp<T>(P.U), st));
  for (int64_t i = 0; i < nsteps; ++i)
    if ((rc = enqueue_step<T>(p, P, s, dt, i + 1 < nsteps, nullptr, st, &pf))) return rc;
  HIT_CK(launch_scatter<T>(vp<T>(P.U), static_cast<V2<T>*>(out), P.g, st));
  HIT_CK(cudaStreamSynchronize(st));
  for (int c = 0; c < HIT_NUM_KERNEL_CLASSES; ++c) {
    ms[c] = 0.0;
    launches[c] = 0;
  }
  for (size_t k = 0; k < pf.cls.size(); ++k) {
    float t = 0.f;
    HIT_CK(cudaEventElapsedTime(&t, pf.ev[2 * k], pf.ev[2 * k + 1]));
    ms[pf.cls[k]] += t;
    launches[pf.cls[k]] += 1;
  }
  return HIT_OK;
}

int check_params(const hit_params* pr) {
  if (!pr) return fail(HIT_E_INVALID, "params is NULL");
  if (pr->forcing_kind < 0 || pr->forcing_kind > 3) return fail(HIT_E_INVALID, "unknown forcing_kind");
  return HIT_OK;
}

// External force f (reference layout) gathered into the path's compact buffer
// FEXT, which the step epilogue adds to the nonlinear term before the mask and
// the projection (the modes outside the 2/3 box of the dealiased path are
// dropped by the gather, which the mask would zero anyway).
template <typename T> int gather_force(hit_plan* p, Path& P, const void* f, cudaStream_t st) {
  int rc;
  if ((rc = ensure(P.FEXT, (size_t)3 * P.g.Mx * P.g.My * P.g.Mzp * sizeof(V2<T>)))) return rc;
  GatherArgs<T> a{};
  a.ext = static_cast<const V2<T>*>(f);
  a.cmp = vp<T>(P.FEXT);
  a.g = P.g;
  a.k = ktab_of<T>(p);
  a.partial = nullptr;
  HIT_CK(launch_gather<T>(a, P.gather_blocks, st));
  return HIT_OK;
}

template <typename T>
int rhs_impl(hit_plan* p, const void* u_hat, const hit_params* pr, void* du, const void* fext, cudaStream_t st) {
  int rc;
  const int which = (pr->flags & HIT_FLAG_ASSUME_DEALIASED) ? 1 : 0;
  if ((rc = ensure_path<T>(p, which))) return rc;
  Path& P = p->path[which];
  const Scalars s = scalars_of(pr);
  if (fext && (rc = gather_force<T>(p, P, fext, st))) return rc;
  if ((rc = gather_state<T>(p, P, u_hat, s, st))) return rc;
  if ((rc = launch_p1_of<T>(p, P, vp<T>(P.U), st))) return rc;
  if ((rc = launch_p2<T>(p, P, st))) return rc;
  if ((rc = launch_p3_stage<T>(p, P, s, 0, 0.0, false, false, fext ? vp<T>(P.FEXT) : nullptr, st))) return rc;
  HIT_CK(launch_scatter<T>(vp<T>(P.D), static_cast<V2<T>*>(du), P.g, st));
  return HIT_OK;
}

// Loop control of the rollout graph: k_loop_set (launched on the caller's
// stream before the graph) stores the count of loop steps, k_loop_arm (the
// graph's first node) opens the while node when it is positive, and
// k_loop_next (the last node of the loop body) counts one step down and
// closes the loop at zero.
__global__ void k_loop_set(long long* left, long long n) { *left = n; }
__global__ void k_loop_arm(cudaGraphConditionalHandle h, const long long* left) {
  cudaGraphSetConditional(h, *left > 0 ? 1u : 0u);
}
__global__ void k_loop_next(cudaGraphConditionalHandle h, long long* left) {
  const long long v = *left - 1;
  *left = v;
  cudaGraphSetConditional(h, v > 0 ? 1u : 0u);
}

// The whole rollout of nsteps >= 1 steps from the x-inverse of U as one graph
// (step(fuse_next, stream) enqueues one step):
//   k_loop_arm -> while (left > 0) { step that ends with the next step's
//   x-inverse; k_loop_next } -> last step.
// The loop count lives in device memory (P.loop), so one instantiated graph
// serves every nsteps: the lax.scan of integrators.py:41-53 without a host
// launch per step.
template <class STEP>
int build_loop_graph(hit_plan* p, Path& P, STEP&& step, cudaGraphExec_t* exec) {
  int rc;
  cudaGraph_t g = nullptr;
  HIT_CK(cudaGraphCreate(&g, 0));
  struct Owner {
    cudaGraph_t g;
    ~Owner() { cudaGraphDestroy(g); }
  } own{g};
  cudaGraphConditionalHandle h;
  HIT_CK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
  long long* left = static_cast<long long*>(P.loop.p);
  cudaGraphNode_t arm = nullptr, loop = nullptr;
  {
    void* args[] = {&h, &left};
    cudaKernelNodeParams kp{};
    kp.func = reinterpret_cast<void*>(&k_loop_arm);
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(1);
    kp.kernelParams = args;
    HIT_CK(cudaGraphAddKernelNode(&arm, g, nullptr, 0, &kp));
  }
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  HIT_CK(cudaGraphAddNode(&loop, g, &arm, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  // loop body: one step that prepares the next, then the count
  HIT_CK(cudaStreamBeginCaptureToGraph(p->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  rc = step(true, p->cap);
  if (!rc) k_loop_next<<<1, 1, 0, p->cap>>>(h, left);
  cudaGraph_t got = nullptr;
  cudaError_t e = cudaStreamEndCapture(p->cap, &got);
  if (rc) return rc;
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "rollout loop body capture");
  // after the loop: the last step
  HIT_CK(cudaStreamBeginCaptureToGraph(p->cap, g, &loop, nullptr, 1, cudaStreamCaptureModeThreadLocal));
  rc = step(false, p->cap);
  e = cudaStreamEndCapture(p->cap, &got);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "rollout last-step capture");
  HIT_CK(cudaGraphInstantiate(exec, g, 0));
  return HIT_OK;
}

template <typename T>
int build_rollout_graph(hit_plan* p, Path& P, const Scalars& s, double dt, const V2<T>* fext,
                        cudaGraphExec_t* exec) {
  return build_loop_graph(
      p, P, [&](bool fuse_next, cudaStream_t cs) { return enqueue_step<T>(p, P, s, dt, fuse_next, fext, cs); },
      exec);
}

template <typename T>
int rollout_impl(hit_plan* p, const void* u_hat, const hit_params* pr, double dt, int64_t nsteps, void* out,
                 const void* fext, cudaStream_t st) {
  int rc;
  const int which = (pr->flags & HIT_FLAG_ASSUME_DEALIASED) ? 1 : 0;
  if ((rc = ensure_path<T>(p, which))) return rc;
  Path& P = p->path[which];
  const Scalars s = scalars_of(pr);
  if (fext && (rc = gather_force<T>(p, P, fext, st))) return rc;
  if ((rc = gather_state<T>(p, P, u_hat, s, st))) return rc;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  HIT_CK(cudaStreamIsCapturing(st, &cs));
  if (nsteps == 1 || (nsteps > 0 && cs != cudaStreamCaptureStatusNone)) {
    // the caller is capturing `st` into its own graph, or a single step (a
    // graph with a conditional node would hide its kernels from per-kernel
    // profilers): enqueue the step kernels themselves
    if ((rc = launch_p1_of<T>(p, P, vp<T>(P.U), st))) return rc;
    for (int64_t i = 0; i < nsteps; ++i)
      if ((rc = enqueue_step<T>(p, P, s, dt, i + 1 < nsteps, fext ? vp<T>(P.FEXT) : nullptr, st))) return rc;
  } else if (nsteps > 0) {
    const GraphKey key{s.nu, s.A, s.eps, pr->kmin, pr->kmax, s.E_target, s.tau, dt, s.forcing, s.ifrk, fext ? 1 : 0};
    if ((rc = ensure(P.loop, sizeof(long long)))) return rc;
    if (!P.key_valid || !(P.key == key)) {
      if (P.exec) cudaGraphExecDestroy(P.exec);
      P.exec = nullptr;
      P.key_valid = false;
      if ((rc = build_rollout_graph<T>(p, P, s, dt, fext ? vp<T>(P.FEXT) : nullptr, &P.exec))) return rc;
      P.key = key;
      P.key_valid = true;
    }
    k_loop_set<<<1, 1, 0, st>>>(static_cast<long long*>(P.loop.p), (long long)(nsteps - 1));
    HIT_CK(cudaGetLastError());
    if ((rc = launch_p1_of<T>(p, P, vp<T>(P.U), st))) return rc;
    HIT_CK(cudaGraphLaunch(P.exec, st));
  }
  HIT_CK(launch_scatter<T>(vp<T>(P.U), static_cast<V2<T>*>(out), P.g, st));
  return HIT_OK;
}

// Coarse-LES rollout with the closure fused into the first stage of every
// step (float32, dealiased path): gather, the LES x-inverse, the steps as one
// graph with a device-side loop (or enqueued into the caller's capture),
// scatter.
int les_rollout_impl(hit_plan* p, const void* u_hat, const hit_params* pr, const hit_mlp_weights& w, int* err,
                     double dt, int64_t nsteps, void* out, cudaStream_t st) {
  int rc;
  if ((rc = ensure_path<float>(p, 1))) return rc;
  Path& P = p->path[1];
  const Scalars s = scalars_of(pr);
  const Geom& g = P.g;
  const size_t V = sizeof(float2);
  if ((rc = ensure(P.t12, (size_t)12 * g.Nx * g.My * g.Mzp * V))) return rc;
  if ((rc = ensure(P.u12, (size_t)12 * g.Nx * g.Ny * g.Mzp * V))) return rc;
  if ((rc = ensure(P.FEXT, (size_t)3 * g.Mx * g.My * g.Mzp * V))) return rc;
  if ((rc = ensure(P.loop, sizeof(long long)))) return rc;
  if ((rc = gather_state<float>(p, P, u_hat, s, st))) return rc;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  HIT_CK(cudaStreamIsCapturing(st, &cs));
  if (nsteps == 1 || (nsteps > 0 && cs != cudaStreamCaptureStatusNone)) {
    if ((rc = launch_p1_of<float>(p, P, vp<float>(P.U), st, true))) return rc;
    for (int64_t i = 0; i < nsteps; ++i)
      if ((rc = enqueue_les_step(p, P, s, dt, i + 1 < nsteps, w, err, st))) return rc;
  } else if (nsteps > 0) {
    const GraphKey key{s.nu, s.A, s.eps, pr->kmin, pr->kmax, s.E_target, s.tau, dt, s.forcing, s.ifrk, 2};
    const bool same_w = std::memcmp(&P.les_w, &w, sizeof(w)) == 0 && P.les_err == err;
    if (!P.les_key_valid || !(P.les_key == key) || !same_w) {
      if (P.les_exec) cudaGraphExecDestroy(P.les_exec);
      P.les_exec = nullptr;
      P.les_key_valid = false;
      if ((rc = build_loop_graph(
               p, P, [&](bool fuse_next, cudaStream_t c) { return enqueue_les_step(p, P, s, dt, fuse_next, w, err, c); },
               &P.les_exec)))
        return rc;
      P.les_key = key;
      P.les_w = w;
      P.les_err = err;
      P.les_key_valid = true;
    }
    k_loop_set<<<1, 1, 0, st>>>(static_cast<long long*>(P.loop.p), (long long)(nsteps - 1));
    HIT_CK(cudaGetLastError());
    if ((rc = launch_p1_of<float>(p, P, vp<float>(P.U), st, true))) return rc;
    HIT_CK(cudaGraphLaunch(P.les_exec, st));
  }
  HIT_CK(launch_scatter<float>(vp<float>(P.U), static_cast<float2*>(out), P.g, st));
  return HIT_OK;
}

template <typename T> int to_physical_impl(hit_plan* p, const void* u_hat, int nc, void* u, cudaStream_t st) {
  const Geom g = make_geom(p->Nx, p->Ny, p->Nz, false);
  int rc;
  if ((rc = ensure(p->xws, (size_t)nc * g.Nx * g.Ny * g.Mzp * sizeof(V2<T>)))) return rc;
  const int Wx = axis_tile_w<T>(g.Nx), Wy = axis_tile_w<T>(g.Ny);
  const long long wc = (long long)g.Nx * g.Ny * g.Mzp;
  AxisArgs<T> a{};
  a.src = static_cast<const V2<T>*>(u_hat);
  a.dst = vp<T>(p->xws);
  a.s_c = (long long)g.Nx * g.Ny * g.Nzh;
  a.s_a = (long long)g.Ny * g.Nzh;
  a.s_o = g.Nzh;
  a.d_c = wc;
  a.d_a = (long long)g.Ny * g.Mzp;
  a.d_o = g.Mzp;
  a.Min = a.Mout = g.Nx;
  a.hin = a.hout = g.Nx / 2;
  a.nz = g.Nzh;
  a.tw = tw_of<T>(p);
  HIT_CK(launch_axis<T>(g.Nx, true, a, (g.Nzh + Wx - 1) / Wx, g.Ny, nc, st));
  AxisArgs<T> b{};
  b.src = vp<T>(p->xws);
  b.dst = vp<T>(p->xws);
  b.s_c = b.d_c = wc;
  b.s_a = b.d_a = g.Mzp;
  b.s_o = b.d_o = (long long)g.Ny * g.Mzp;
  b.Min = b.Mout = g.Ny;
  b.hin = b.hout = g.Ny / 2;
  b.nz = g.Nzh;
  b.src_cols = g.Mzp;  // padded rows: staged whole tiles
  b.tw = tw_of<T>(p);
  HIT_CK(launch_axis<T>(g.Ny, true, b, (g.Nzh + Wy - 1) / Wy, g.Nx, nc, st));
  ZRealArgs<T> z{};
  z.cbuf = vp<T>(p->xws);
  z.rbuf = static_cast<T*>(u);
  z.cc_stride = wc;
  z.rc_stride = (long long)g.Nx * g.Ny * g.Nz;
  z.nrows = g.Nx * g.Ny;
  z.Mz = g.Nzh;
  z.Mzp = g.Mzp;
  z.scale = (T)(1.0 / ((double)g.Nx * g.Ny * g.Nz));
  z.tw = tw_of<T>(p);
  HIT_CK(launch_zc2r<T>(g.H, z, nc, st));
  return HIT_OK;
}

template <typename T> int to_spectral_impl(hit_plan* p, const void* u, int nc, void* u_hat, cudaStream_t st) {
  const Geom g = make_geom(p->Nx, p->Ny, p->Nz, false);
  int rc;
  if ((rc = ensure(p->xws, (size_t)nc * g.Nx * g.Ny * g.Mzp * sizeof(V2<T>)))) return rc;
  const int Wx = axis_tile_w<T>(g.Nx), Wy = axis_tile_w<T>(g.Ny);
  const long long wc = (long long)g.Nx * g.Ny * g.Mzp;
  ZRealArgs<T> z{};
  z.cbuf = vp<T>(p->xws);
  z.rbuf = const_cast<T*>(static_cast<const T*>(u));
  z.cc_stride = wc;
  z.rc_stride = (long long)g.Nx * g.Ny * g.Nz;
  z.nrows = g.Nx * g.Ny;
  z.Mz = g.Nzh;
  z.Mzp = g.Mzp;
  z.scale = T(1);
  z.tw = tw_of<T>(p);
  HIT_CK(launch_zr2c<T>(g.H, z, nc, st));
  AxisArgs<T> b{};
  b.src = vp<T>(p->xws);
  b.dst = vp<T>(p->xws);
  b.s_c = b.d_c = wc;
  b.s_a = b.d_a = g.Mzp;
  b.s_o = b.d_o = (long long)g.Ny * g.Mzp;
  b.Min = b.Mout = g.Ny;
  b.hin = b.hout = g.Ny / 2;
  b.nz = g.Nzh;
  b.src_cols = g.Mzp;  // padded rows: staged whole tiles
  b.tw = tw_of<T>(p);
  HIT_CK(launch_axis<T>(g.Ny, false, b, (g.Nzh + Wy - 1) / Wy, g.Nx, nc, st));
  AxisArgs<T> a{};
  a.src = vp<T>(p->xws);
  a.dst = static_cast<V2<T>*>(u_hat);
  a.s_c = wc;
  a.s_a = (long long)g.Ny * g.Mzp;
  a.s_o = g.Mzp;
  a.d_c = (long long)g.Nx * g.Ny * g.Nzh;
  a.d_a = (long long)g.Ny * g.Nzh;
  a.d_o = g.Nzh;
  a.Min = a.Mout = g.Nx;
  a.hin = a.hout = g.Nx / 2;
  a.nz = g.Nzh;
  a.src_cols = g.Mzp;  // reads the padded rows of the workspace
  a.tw = tw_of<T>(p);
  HIT_CK(launch_axis<T>(g.Nx, false, a, (g.Nzh + Wx - 1) / Wx, g.Ny, nc, st));
  return HIT_OK;
}

// One axis of the 3-D transform on reference-layout arrays (ncomp, Nx, Ny,
// Nzh), unnormalised: axis 0 / 1 complex along x / y (in and out distinct,
// same layout); axis 2 the real transform along z between (ncomp, Nx, Ny, Nzh)
// complex and (ncomp, Nx, Ny, Nz) real (c2r when inverse: the imaginary parts
// of the kz = 0 and Nyquist entries are dropped), through the padded workspace.
template <typename T>
int axis_fft_impl(hit_plan* p, const void* in, void* out, int nc, int axis, int inverse, cudaStream_t st) {
  const Geom g = make_geom(p->Nx, p->Ny, p->Nz, false);
  const bool inv = inverse != 0;
  if (axis == 0 || axis == 1) {
    const int N = axis == 0 ? g.Nx : g.Ny;
    const int W = axis_tile_w<T>(N);
    AxisArgs<T> a{};
    a.src = static_cast<const V2<T>*>(in);
    a.dst = static_cast<V2<T>*>(out);
    a.s_c = a.d_c = (long long)g.Nx * g.Ny * g.Nzh;
    a.s_a = a.d_a = axis == 0 ? (long long)g.Ny * g.Nzh : g.Nzh;
    a.s_o = a.d_o = axis == 0 ? g.Nzh : (long long)g.Ny * g.Nzh;
    a.Min = a.Mout = N;
    a.hin = a.hout = N / 2;
    a.nz = g.Nzh;
    a.tw = tw_of<T>(p);
    HIT_CK(launch_axis<T>(N, inv, a, (g.Nzh + W - 1) / W, axis == 0 ? g.Ny : g.Nx, nc, st));
    return HIT_OK;
  }
  int rc;
  if ((rc = ensure(p->xws, (size_t)nc * g.Nx * g.Ny * g.Mzp * sizeof(V2<T>)))) return rc;
  const size_t es = sizeof(V2<T>);
  const size_t rows = (size_t)nc * g.Nx * g.Ny;
  ZRealArgs<T> z{};
  z.cbuf = vp<T>(p->xws);
  z.cc_stride = (long long)g.Nx * g.Ny * g.Mzp;
  z.rc_stride = (long long)g.Nx * g.Ny * g.Nz;
  z.nrows = g.Nx * g.Ny;
  z.Mz = g.Nzh;
  z.Mzp = g.Mzp;
  z.scale = T(1);
  z.tw = tw_of<T>(p);
  if (inv) {
    HIT_CK(cudaMemcpy2DAsync(p->xws.p, g.Mzp * es, in, g.Nzh * es, g.Nzh * es, rows, cudaMemcpyDeviceToDevice, st));
    z.rbuf = static_cast<T*>(out);
    HIT_CK(launch_zc2r<T>(g.H, z, nc, st));
  } else {
    z.rbuf = const_cast<T*>(static_cast<const T*>(in));
    HIT_CK(launch_zr2c<T>(g.H, z, nc, st));
    HIT_CK(cudaMemcpy2DAsync(out, g.Nzh * es, p->xws.p, g.Mzp * es, g.Nzh * es, rows, cudaMemcpyDeviceToDevice, st));
  }
  return HIT_OK;
}

// spectrum / budget over the reference layout
template <typename T>
int diag_impl(hit_plan* p, const void* u_hat, const hit_params* pr, double* E, double* Ec, double* budget,
              cudaStream_t st) {
  const Geom g = make_geom(p->Nx, p->Ny, p->Nz, false);
  const int nshell = (E || Ec) ? p->smax + 1 : 0;
  const int nv = 3 * nshell + NSCAL;
  int rc;
  if ((rc = ensure(p->dpartial, (size_t)p->diag_blocks * nv * sizeof(double)))) return rc;
  if ((rc = ensure(p->dsums, (size_t)nv * sizeof(double)))) return rc;
  Scalars s{};
  if (pr) s = scalars_of(pr);
  ModeSumArgs<T> a{};
  a.u = static_cast<const V2<T>*>(u_hat);
  a.c_c = (long long)g.Nx * g.Ny * g.Nzh;
  a.c_x = (long long)g.Ny * g.Nzh;
  a.c_y = g.Nzh;
  a.g = g;
  a.k = ktab_of<T>(p);
  a.kmin2 = (T)s.kmin2;
  a.kmax2 = (T)s.kmax2;
  a.k0 = (T)(2.0 * M_PI / p->Lx);
  a.nshell = nshell;
  a.partial = static_cast<double*>(p->dpartial.p);
  HIT_CK(launch_mode_sums<T>(a, p->diag_blocks, st));
  SumArgs sa{static_cast<const double*>(p->dpartial.p), p->diag_blocks, nv, static_cast<double*>(p->dsums.p)};
  HIT_CK(launch_finalize_sums(sa, st));
  BudgetArgs b{};
  b.sums = static_cast<const double*>(p->dsums.p);
  b.nshell = nshell;
  b.spec = E;
  b.comp = Ec;
  b.budget = budget;
  b.forcing = pr ? s.forcing : 0;
  b.ntot2 = ntot2_of(p);
  b.nu = s.nu;
  b.A = s.A;
  b.eps = s.eps;
  b.E_target = s.E_target;
  b.tau = s.tau;
  b.tiny = tiny_of<T>();
  HIT_CK(launch_finalize_budget(b, st));
  return HIT_OK;
}

// ---------------------------------------------------------------------------
// discrete adjoint (general path, reference layout): RHS transpose, RK4 step
// transpose (stage inputs recomputed), rollout transpose with checkpoints
// ---------------------------------------------------------------------------

template <typename T> int adj_blocks(const hit_plan* p) {
  const long long nm = (long long)p->Nx * p->Ny * (p->Nz / 2 + 1);
  return (int)std::min<long long>((nm + NT - 1) / NT, 8 * 148);
}

// ub = (d rhs / d u)^T v at u; the parameter cotangents (nu, A, eps) are added
// to pct (device).
template <typename T>
int rhs_vjp_impl(hit_plan* p, const V2<T>* u, const Scalars& s, const V2<T>* v, V2<T>* ub, double* pct,
                 cudaStream_t st) {
  const Geom g = make_geom(p->Nx, p->Ny, p->Nz, false);
  const long long nm = (long long)g.Nx * g.Ny * g.Nzh, n3 = (long long)g.Nx * g.Ny * g.Nz;
  const int nb = adj_blocks<T>(p);
  int rc;
  if ((rc = ensure(p->ax9, 9 * nm * sizeof(V2<T>)))) return rc;
  if ((rc = ensure(p->aph, 9 * n3 * sizeof(T)))) return rc;
  if ((rc = ensure(p->as6, 6 * nm * sizeof(V2<T>)))) return rc;
  if ((rc = ensure(p->apart, (size_t)nb * 6 * sizeof(double)))) return rc;
  if ((rc = ensure(p->asums, 6 * sizeof(double)))) return rc;
  if ((rc = ensure(p->ascal, 8 * sizeof(double)))) return rc;
  AdjArgs<T> a{};
  a.u = u;
  a.v = v;
  a.x9 = vp<T>(p->ax9);
  a.s6 = vp<T>(p->as6);
  a.ub = ub;
  a.scal = static_cast<const double*>(p->ascal.p);
  a.partial = static_cast<double*>(p->apart.p);
  a.g = g;
  a.k = ktab_of<T>(p);
  a.nu = (T)s.nu;
  a.kmin2 = (T)s.kmin2;
  a.kmax2 = (T)s.kmax2;
  HIT_CK(launch_adj_sums<T>(a, nb, st));
  SumArgs sa{static_cast<const double*>(p->apart.p), nb, 6, static_cast<double*>(p->asums.p)};
  HIT_CK(launch_finalize_sums(sa, st));
  AdjCoefArgs c{};
  c.sums = static_cast<const double*>(p->asums.p);
  c.scal = static_cast<double*>(p->ascal.p);
  c.pct = pct;
  c.forcing = s.forcing;
  c.ntot2 = ntot2_of(p);
  c.nu = s.nu;
  c.A = s.A;
  c.eps = s.eps;
  c.E_target = s.E_target;
  c.tau = s.tau;
  c.tiny = tiny_of<T>();
  HIT_CK(launch_adj_coef(c, st));
  HIT_CK(launch_adj_prep<T>(a, st));
  if ((rc = to_physical_impl<T>(p, p->ax9.p, 9, p->aph.p, st))) return rc;
  HIT_CK(launch_adj_cross<T>(static_cast<T*>(p->aph.p), n3, st));
  if ((rc = to_spectral_impl<T>(p, static_cast<T*>(p->aph.p) + 3 * n3, 6, p->as6.p, st))) return rc;
  HIT_CK(launch_adj_combine<T>(a, st));
  return HIT_OK;
}

hit_params general_params(const hit_params* pr) {
  hit_params q = *pr;
  q.flags &= ~(unsigned)HIT_FLAG_ASSUME_DEALIASED;  // recompute on the general path
  return q;
}

// ub_out = (d rk4_step / d u)^T ub_in at u (stage inputs recomputed); ub_out
// may alias ub_in.
// With fext (reference layout) the step holds that force over its four
// stages (rk4_step(..., f_ext=), the LES step), and fbar (nullable) receives
// the force's cotangent: every stage adds P f (P = dealias + projection), so
// fbar = P (sum of the stages' cotangents).
template <typename T>
int rk4_vjp_impl(hit_plan* p, const V2<T>* u, const hit_params* pr, double dt, const V2<T>* ub_in, V2<T>* ub_out,
                 double* pct, cudaStream_t st, const void* fext = nullptr, V2<T>* fbar = nullptr) {
  const long long n = 3LL * p->Nx * p->Ny * (p->Nz / 2 + 1);
  const size_t bytes = n * sizeof(V2<T>);
  int rc;
  for (Buf* b : {&p->ast[0], &p->ast[1], &p->ast[2], &p->ak, &p->akb, &p->asb, &p->aacc})
    if ((rc = ensure(*b, bytes))) return rc;
  const hit_params pg = general_params(pr);
  const Scalars s = scalars_of(pr);
  V2<T>* S2 = vp<T>(p->ast[0]);
  V2<T>* S3 = vp<T>(p->ast[1]);
  V2<T>* S4 = vp<T>(p->ast[2]);
  V2<T>* K = vp<T>(p->ak);
  V2<T>* KB = vp<T>(p->akb);
  V2<T>* SB = vp<T>(p->asb);
  V2<T>* ACC = vp<T>(p->aacc);
  const T h = (T)(0.5 * dt), d = (T)dt, d3 = (T)(dt / 3.0), d6 = (T)(dt / 6.0);
  V2<T>* FB = nullptr;
  if (fbar) {
    if ((rc = ensure(p->afb, bytes))) return rc;
    FB = vp<T>(p->afb);
  }
  // the stages' cotangents summed into FB (first one: FB = KB)
  auto add_fb = [&](bool first) -> int {
    if (FB) HIT_CK(launch_axpby<T>(KB, T(1), first ? nullptr : FB, first ? T(0) : T(1), FB, n, st));
    return HIT_OK;
  };
  // stage inputs (integrators.py:32-38)
  if ((rc = rhs_impl<T>(p, u, &pg, K, fext, st))) return rc;
  HIT_CK(launch_axpby<T>(u, T(1), K, h, S2, n, st));
  if ((rc = rhs_impl<T>(p, S2, &pg, K, fext, st))) return rc;
  HIT_CK(launch_axpby<T>(u, T(1), K, h, S3, n, st));
  if ((rc = rhs_impl<T>(p, S3, &pg, K, fext, st))) return rc;
  HIT_CK(launch_axpby<T>(u, T(1), K, d, S4, n, st));
  // transpose of u + dt/6 (k1 + 2 k2 + 2 k3 + k4), stage by stage backwards
  HIT_CK(launch_axpby<T>(ub_in, d6, nullptr, T(0), KB, n, st));
  if ((rc = add_fb(true))) return rc;
  if ((rc = rhs_vjp_impl<T>(p, S4, s, KB, SB, pct, st))) return rc;
  HIT_CK(launch_axpby<T>(ub_in, T(1), SB, T(1), ACC, n, st));
  HIT_CK(launch_axpby<T>(ub_in, d3, SB, d, KB, n, st));
  if ((rc = add_fb(false))) return rc;
  if ((rc = rhs_vjp_impl<T>(p, S3, s, KB, SB, pct, st))) return rc;
  HIT_CK(launch_axpby<T>(ACC, T(1), SB, T(1), ACC, n, st));
  HIT_CK(launch_axpby<T>(ub_in, d3, SB, h, KB, n, st));
  if ((rc = add_fb(false))) return rc;
  if ((rc = rhs_vjp_impl<T>(p, S2, s, KB, SB, pct, st))) return rc;
  HIT_CK(launch_axpby<T>(ACC, T(1), SB, T(1), ACC, n, st));
  HIT_CK(launch_axpby<T>(ub_in, d6, SB, h, KB, n, st));
  if ((rc = add_fb(false))) return rc;
  if ((rc = rhs_vjp_impl<T>(p, u, s, KB, SB, pct, st))) return rc;
  HIT_CK(launch_axpby<T>(ACC, T(1), SB, T(1), ub_out, n, st));
  if (fbar) {
    const Geom g = make_geom(p->Nx, p->Ny, p->Nz, false);
    HIT_CK(launch_dealias_project<T>(FB, fbar, g, ktab_of<T>(p), 1, 1, st));
  }
  return HIT_OK;
}

// u0_bar = (d rollout / d u0)^T ub at u0: states every K steps are kept (the
// forward runs as graph-replayed steps), each segment is recomputed forwards
// and transposed step by step backwards.
template <typename T>
int rollout_vjp_impl(hit_plan* p, const void* u0, const hit_params* pr, double dt, int64_t nsteps, int K,
                     const void* ub, void* u0_bar, double* pct, cudaStream_t st) {
  const long long n = 3LL * p->Nx * p->Ny * (p->Nz / 2 + 1);
  const size_t bytes = n * sizeof(V2<T>);
  const int64_t nseg = (nsteps + K - 1) / K;
  int rc;
  if ((rc = ensure(p->ack, std::max<int64_t>(nseg, 1) * bytes))) return rc;
  if ((rc = ensure(p->aseg, (size_t)K * bytes))) return rc;
  if ((rc = ensure(p->aub, bytes))) return rc;
  const hit_params pg = general_params(pr);
  V2<T>* CK = vp<T>(p->ack);
  V2<T>* SEG = vp<T>(p->aseg);
  V2<T>* UB = vp<T>(p->aub);
  HIT_CK(cudaMemcpyAsync(UB, ub, bytes, cudaMemcpyDeviceToDevice, st));
  if (nsteps == 0) {
    HIT_CK(cudaMemcpyAsync(u0_bar, UB, bytes, cudaMemcpyDeviceToDevice, st));
    return HIT_OK;
  }
  HIT_CK(cudaMemcpyAsync(CK, u0, bytes, cudaMemcpyDeviceToDevice, st));
  for (int64_t j = 1; j < nseg; ++j)
    if ((rc = rollout_impl<T>(p, CK + (j - 1) * n, &pg, dt, K, CK + j * n, nullptr, st))) return rc;
  for (int64_t j = nseg - 1; j >= 0; --j) {
    const int len = (int)std::min<int64_t>(K, nsteps - j * K);
    HIT_CK(cudaMemcpyAsync(SEG, CK + j * n, bytes, cudaMemcpyDeviceToDevice, st));
    for (int i = 1; i < len; ++i)
      if ((rc = rollout_impl<T>(p, SEG + (i - 1) * n, &pg, dt, 1, SEG + i * n, nullptr, st))) return rc;
    for (int i = len - 1; i >= 0; --i)
      if ((rc = rk4_vjp_impl<T>(p, SEG + i * n, pr, dt, UB, UB, pct, st))) return rc;
  }
  HIT_CK(cudaMemcpyAsync(u0_bar, UB, bytes, cudaMemcpyDeviceToDevice, st));
  return HIT_OK;
}

// entry-point wrappers: zero the parameter cotangents, run, copy them out
template <typename T>
int vjp_entry(hit_plan* p, int which, const void* u, const hit_params* pr, double dt, int64_t nsteps, int K,
              const void* ct, void* ubar, double* pct_out, cudaStream_t st) {
  int rc;
  if ((rc = ensure(p->apct, 4 * sizeof(double)))) return rc;
  double* pct = static_cast<double*>(p->apct.p);
  HIT_CK(cudaMemsetAsync(pct, 0, 4 * sizeof(double), st));
  const V2<T>* uu = static_cast<const V2<T>*>(u);
  const V2<T>* cc = static_cast<const V2<T>*>(ct);
  V2<T>* ub = static_cast<V2<T>*>(ubar);
  if (which == 0) rc = rhs_vjp_impl<T>(p, uu, scalars_of(pr), cc, ub, pct, st);
  else if (which == 1) rc = rk4_vjp_impl<T>(p, uu, pr, dt, cc, ub, pct, st);
  else rc = rollout_vjp_impl<T>(p, u, pr, dt, nsteps, K, ct, ubar, pct, st);
  if (rc) return rc;
  if (pct_out) HIT_CK(cudaMemcpyAsync(pct_out, pct, 3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
  return HIT_OK;
}

template <typename T>
int forced_vjp_entry(hit_plan* p, const void* u, const hit_params* pr, const void* f, double dt, const void* ct,
                     void* ubar, void* fbar, double* pct_out, cudaStream_t st) {
  int rc;
  if ((rc = ensure(p->apct, 4 * sizeof(double)))) return rc;
  double* pct = static_cast<double*>(p->apct.p);
  HIT_CK(cudaMemsetAsync(pct, 0, 4 * sizeof(double), st));
  if ((rc = rk4_vjp_impl<T>(p, static_cast<const V2<T>*>(u), pr, dt, static_cast<const V2<T>*>(ct),
                            static_cast<V2<T>*>(ubar), pct, st, f, static_cast<V2<T>*>(fbar))))
    return rc;
  if (pct_out) HIT_CK(cudaMemcpyAsync(pct_out, pct, 3 * sizeof(double), cudaMemcpyDeviceToDevice, st));
  return HIT_OK;
}

// tau_bar (physical, 6 x N^3) = cotangent of the stress whose sgs force has
// cotangent f_bar (transposes of hit_sgs_force and of the stress's rfftn)
template <typename T> int sgs_force_vjp_impl(hit_plan* p, const void* fbar, void* tbar, cudaStream_t st) {
  const Geom g = make_geom(p->Nx, p->Ny, p->Nz, false);
  int rc;
  if ((rc = ensure(p->ax9, 9 * (size_t)g.Nx * g.Ny * g.Nzh * sizeof(V2<T>)))) return rc;
  HIT_CK(launch_sgs_force_vjp<T>(static_cast<const V2<T>*>(fbar), vp<T>(p->ax9), g, ktab_of<T>(p),
                                 (T)((double)p->Nx * p->Ny * p->Nz), st));
  return to_physical_impl<T>(p, p->ax9.p, 6, tbar, st);
}

// u_bar += cotangent of u_hat whose velocity gradients have cotangent g_bar
template <typename T> int grad_vjp_impl(hit_plan* p, const void* gbar, void* ubar, cudaStream_t st) {
  const Geom g = make_geom(p->Nx, p->Ny, p->Nz, false);
  int rc;
  if ((rc = ensure(p->ax9, 9 * (size_t)g.Nx * g.Ny * g.Nzh * sizeof(V2<T>)))) return rc;
  if ((rc = to_spectral_impl<T>(p, gbar, 9, p->ax9.p, st))) return rc;
  HIT_CK(launch_grad9_vjp<T>(vp<T>(p->ax9), static_cast<V2<T>*>(ubar), g, ktab_of<T>(p),
                             (T)(1.0 / ((double)p->Nx * p->Ny * p->Nz)), st));
  return HIT_OK;
}

template <typename T> void fill_tables(hit_plan* p, std::string& kt, std::string& tw) {
  const double two_pi = 2.0 * M_PI;
  const int Nzh = p->Nz / 2 + 1;
  kt.resize(sizeof(T) * (p->Nx + p->Ny + Nzh));
  T* k = reinterpret_cast<T*>(&kt[0]);
  auto freq = [](int i, int n) { return i < n / 2 ? i : i - n; };
  for (int i = 0; i < p->Nx; ++i) k[i] = (T)(two_pi / p->Lx * (double)freq(i, p->Nx));
  for (int i = 0; i < p->Ny; ++i) k[p->Nx + i] = (T)(two_pi / p->Ly * (double)freq(i, p->Ny));
  for (int i = 0; i < Nzh; ++i) k[p->Nx + p->Ny + i] = (T)(two_pi / p->Lz * (double)i);
  tw.resize(sizeof(V2<T>) * TWN);
  V2<T>* w = reinterpret_cast<V2<T>*>(&tw[0]);
  const long double pi = acosl(-1.0L);
  for (int m = 0; m < TWN; ++m) {
    const long double th = 2.0L * pi * (long double)m / (long double)TWN;
    long double c = cosl(th), sn = -sinl(th);
    if (fabsl(c) < 1e-30L) c = 0.0L;
    if (fabsl(sn) < 1e-30L) sn = 0.0L;
    w[m].x = (T)c;
    w[m].y = (T)sn;
  }
}

template <typename T> int create_impl(hit_plan* p) {
  std::string kt, tw;
  fill_tables<T>(p, kt, tw);
  int rc;
  if ((rc = ensure(p->ktab, kt.size()))) return rc;
  if ((rc = ensure(p->tw, tw.size()))) return rc;
  HIT_CK(cudaMemcpy(p->ktab.p, kt.data(), kt.size(), cudaMemcpyHostToDevice));
  HIT_CK(cudaMemcpy(p->tw.p, tw.data(), tw.size(), cudaMemcpyHostToDevice));
  HIT_CK(prepare_fft_kernels<T>(p->Nx, p->Ny, p->Nz));
  return HIT_OK;
}

}  // namespace

namespace hit {
// Sets the thread's last-error string for entry points defined in other files.
int record_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace hit

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

#define DISPATCH(p, call)                                   \
  ((p)->dtype == HIT_DTYPE_F32 ? call<float> : call<double>)

extern "C" {

const char* hit_last_error_string(void) { return g_last_error.c_str(); }

int hit_plan_create(int nx, int ny, int nz, double lx, double ly, double lz, int dtype, hit_plan** out) {
  if (!out) return fail(HIT_E_INVALID, "out is NULL");
  *out = nullptr;
  if (!pow2_ok(nx) || !pow2_ok(ny) || !pow2_ok(nz))
    return fail(HIT_E_UNSUPPORTED, "grid sizes must be powers of two in [4, 1024], got " + std::to_string(nx) + "x" +
                                       std::to_string(ny) + "x" + std::to_string(nz));
  if (dtype != HIT_DTYPE_F32 && dtype != HIT_DTYPE_F64) return fail(HIT_E_UNSUPPORTED, "dtype must be F32 or F64");
  if (!(lx > 0) || !(ly > 0) || !(lz > 0)) return fail(HIT_E_INVALID, "box lengths must be positive");
  hit_plan* p = new hit_plan();
  p->dtype = dtype;
  p->Nx = nx;
  p->Ny = ny;
  p->Nz = nz;
  p->Lx = lx;
  p->Ly = ly;
  p->Lz = lz;
  cudaError_t e = cudaGetDevice(&p->device);
  if (e != cudaSuccess) {
    delete p;
    return cuda_fail(e, "cudaGetDevice");
  }
  const int nmax = std::max(nx, std::max(ny, nz));
  p->smax = (int)std::ceil(std::sqrt(3.0) * nmax / 2.0) + 1;
  const long long nm = (long long)nx * ny * (nz / 2 + 1);
  {
    // k_mode_sums: 4-warp blocks with per-warp compensated bins (2 x 4 x 3 x
    // (smax + 1) doubles), as many resident per SM as their shared memory
    // allows (at most 8), one resident wave
    const long long bins_bytes = 2LL * 4 * 3 * (p->smax + 1) * 8;
    const long long per_sm = std::max(1LL, std::min(8LL, (220LL * 1024) / (bins_bytes + 1024)));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device);
    p->diag_blocks = (int)std::min<long long>((nm + 127) / 128, per_sm * sms);
  }
  int rc = dtype == HIT_DTYPE_F32 ? create_impl<float>(p) : create_impl<double>(p);
  if (rc == HIT_OK) {
    e = cudaStreamCreateWithFlags(&p->cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking);
    for (int k = 0; k < 4 && e == cudaSuccess; ++k) {
      e = cudaEventCreateWithFlags(&p->ev_fork[k], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->ev_join[k], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaStreamCreate / cudaEventCreate");
  }
  if (rc != HIT_OK) {
    hit_plan_destroy(p);
    return rc;
  }
  *out = p;
  return HIT_OK;
}

int hit_plan_destroy(hit_plan* p) {
  if (!p) return HIT_OK;
  DeviceGuard dg(p->device);
  for (Path& P : p->path) {
    if (P.exec) cudaGraphExecDestroy(P.exec);
    if (P.les_exec) cudaGraphExecDestroy(P.les_exec);
    release(P.loop);
    release(P.t12);
    release(P.u12);
    release(P.t6);
    release(P.u6);
    release(P.U);
    release(P.ACC);
    release(P.S);
    release(P.D);
    release(P.partial);
    release(P.coef);
  }
  release(p->ktab);
  release(p->tw);
  release(p->xws);
  release(p->dpartial);
  release(p->dsums);
  for (Buf* b : {&p->ax9, &p->aph, &p->as6, &p->apart, &p->asums, &p->ascal, &p->apct, &p->ast[0], &p->ast[1],
                 &p->ast[2], &p->ak, &p->akb, &p->asb, &p->aacc, &p->aub, &p->ack, &p->aseg, &p->afb})
    release(*b);
  if (p->cap) cudaStreamDestroy(p->cap);
  if (p->side) cudaStreamDestroy(p->side);
  for (int k = 0; k < 4; ++k) {
    if (p->ev_fork[k]) cudaEventDestroy(p->ev_fork[k]);
    if (p->ev_join[k]) cudaEventDestroy(p->ev_join[k]);
  }
  delete p;
  return HIT_OK;
}

int hit_plan_num_shells(const hit_plan* p) { return p ? p->smax : 0; }

int hit_to_physical(hit_plan* p, const void* u_hat, int nc, void* u, void* stream) {
  if (!p || !u_hat || !u) return fail(HIT_E_INVALID, "NULL argument");
  if (nc < 1 || nc > 9) return fail(HIT_E_INVALID, "ncomp must be in [1, 9]");
  DeviceGuard dg(p->device);
  return DISPATCH(p, to_physical_impl)(p, u_hat, nc, u, (cudaStream_t)stream);
}

int hit_to_spectral(hit_plan* p, const void* u, int nc, void* u_hat, void* stream) {
  if (!p || !u_hat || !u) return fail(HIT_E_INVALID, "NULL argument");
  if (nc < 1 || nc > 9) return fail(HIT_E_INVALID, "ncomp must be in [1, 9]");
  DeviceGuard dg(p->device);
  return DISPATCH(p, to_spectral_impl)(p, u, nc, u_hat, (cudaStream_t)stream);
}

int hit_dealias_project(hit_plan* p, const void* u_hat, int dd, int pp, void* out, void* stream) {
  if (!p || !u_hat || !out) return fail(HIT_E_INVALID, "NULL argument");
  DeviceGuard dg(p->device);
  const Geom g = make_geom(p->Nx, p->Ny, p->Nz, false);
  cudaError_t e;
  if (p->dtype == HIT_DTYPE_F32)
    e = launch_dealias_project<float>(static_cast<const float2*>(u_hat), static_cast<float2*>(out), g,
                                      ktab_of<float>(p), dd, pp, (cudaStream_t)stream);
  else
    e = launch_dealias_project<double>(static_cast<const double2*>(u_hat), static_cast<double2*>(out), g,
                                       ktab_of<double>(p), dd, pp, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "dealias_project");
  return HIT_OK;
}

int hit_shell_scale(hit_plan* p, const void* u_hat, const double* c, void* out, void* stream) {
  if (!p || !u_hat || !c || !out) return fail(HIT_E_INVALID, "NULL argument");
  DeviceGuard dg(p->device);
  const Geom g = make_geom(p->Nx, p->Ny, p->Nz, false);
  const double k0 = 2.0 * M_PI / p->Lx;
  cudaError_t e =
      p->dtype == HIT_DTYPE_F32
          ? launch_shell_scale<float>(static_cast<const float2*>(u_hat), static_cast<float2*>(out), g, ktab_of<float>(p),
                                      (float)k0, c, p->smax, (cudaStream_t)stream)
          : launch_shell_scale<double>(static_cast<const double2*>(u_hat), static_cast<double2*>(out), g,
                                       ktab_of<double>(p), k0, c, p->smax, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "shell_scale");
  return HIT_OK;
}

int hit_check_dealiased(hit_plan* p, const void* u_hat, int* flag, void* stream) {
  if (!p || !u_hat || !flag) return fail(HIT_E_INVALID, "NULL argument");
  DeviceGuard dg(p->device);
  const Geom g = make_geom(p->Nx, p->Ny, p->Nz, true);
  cudaError_t e = p->dtype == HIT_DTYPE_F32
                      ? launch_check_box<float>(static_cast<const float2*>(u_hat), g, flag, (cudaStream_t)stream)
                      : launch_check_box<double>(static_cast<const double2*>(u_hat), g, flag, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "check_dealiased");
  return HIT_OK;
}

int hit_rhs(hit_plan* p, const void* u_hat, const hit_params* pr, double t, void* du, void* stream) {
  (void)t;  // no forcing of the reference depends on t
  if (!p || !u_hat || !du) return fail(HIT_E_INVALID, "NULL argument");
  int rc;
  if ((rc = check_params(pr))) return rc;
  DeviceGuard dg(p->device);
  return DISPATCH(p, rhs_impl)(p, u_hat, pr, du, nullptr, (cudaStream_t)stream);
}

int hit_device_status(int* status) {
  if (!status) return fail(HIT_E_INVALID, "NULL argument");
  int z = 0;
  cudaError_t e = take_axis_timeout(status);
  if (e == cudaSuccess) e = take_z_timeout(&z);
  if (e != cudaSuccess) return cuda_fail(e, "device_status");
  *status = *status || z;
  return HIT_OK;
}

int hit_set_wait_limit(int polls) {
  cudaError_t e = set_axis_wait_limit(polls);
  if (e == cudaSuccess) e = set_z_wait_limit(polls);
  return e == cudaSuccess ? HIT_OK : cuda_fail(e, "set_wait_limit");
}

int hit_rhs_forced(hit_plan* p, const void* u_hat, const hit_params* pr, const void* f_ext, double t, void* du,
                   void* stream) {
  (void)t;
  if (!p || !u_hat || !f_ext || !du) return fail(HIT_E_INVALID, "NULL argument");
  int rc;
  if ((rc = check_params(pr))) return rc;
  DeviceGuard dg(p->device);
  return DISPATCH(p, rhs_impl)(p, u_hat, pr, du, f_ext, (cudaStream_t)stream);
}

int hit_rollout_forced(hit_plan* p, const void* u_hat, const hit_params* pr, const void* f_ext, double dt,
                       int64_t nsteps, double t0, void* out, void* stream) {
  (void)t0;
  if (!p || !u_hat || !f_ext || !out) return fail(HIT_E_INVALID, "NULL argument");
  if (nsteps < 0) return fail(HIT_E_INVALID, "nsteps must be >= 0");
  int rc;
  if ((rc = check_params(pr))) return rc;
  DeviceGuard dg(p->device);
  return DISPATCH(p, rollout_impl)(p, u_hat, pr, dt, nsteps, out, f_ext, (cudaStream_t)stream);
}

int hit_rk4_step(hit_plan* p, const void* u_hat, const hit_params* pr, double dt, double t, void* out, void* stream) {
  (void)t;
  if (!p || !u_hat || !out) return fail(HIT_E_INVALID, "NULL argument");
  int rc;
  if ((rc = check_params(pr))) return rc;
  DeviceGuard dg(p->device);
  return DISPATCH(p, rollout_impl)(p, u_hat, pr, dt, 1, out, nullptr, (cudaStream_t)stream);
}

int hit_les_rollout(hit_plan* p, const void* u_hat, const hit_params* pr, const hit_mlp_weights* w, double dt,
                    int64_t nsteps, void* out, int* err_dev, void* stream) {
  if (!p || !u_hat || !pr || !w || !out || !err_dev) return fail(HIT_E_INVALID, "NULL argument");
  if (!w->w1t || !w->w2t || !w->w3t || !w->w4t || !w->b2 || !w->b3 || !w->b4)
    return fail(HIT_E_INVALID, "les_rollout: NULL MLP weight");
  if (nsteps < 0) return fail(HIT_E_INVALID, "nsteps must be >= 0");
  int rc;
  if ((rc = check_params(pr))) return rc;
  if (p->dtype != HIT_DTYPE_F32) return fail(HIT_E_UNSUPPORTED, "les_rollout: float32 plans only");
  if (!(pr->flags & HIT_FLAG_ASSUME_DEALIASED))
    return fail(HIT_E_UNSUPPORTED, "les_rollout: the state must be dealiased (HIT_FLAG_ASSUME_DEALIASED)");
  if (pr->flags & HIT_FLAG_INTEGRATING_FACTOR) return fail(HIT_E_UNSUPPORTED, "les_rollout: RK4 only");
  if (p->Nx > 256 || !zles_supported(p->Nz))
    return fail(HIT_E_UNSUPPORTED, "les_rollout: needs Nx <= 256 and Nz in {32, 64, 128}");
  DeviceGuard dg(p->device);
  return les_rollout_impl(p, u_hat, pr, *w, err_dev, dt, nsteps, out, (cudaStream_t)stream);
}

int hit_rollout(hit_plan* p, const void* u_hat, const hit_params* pr, double dt, int64_t nsteps, double t0, void* out,
                void* stream) {
  (void)t0;
  if (!p || !u_hat || !out) return fail(HIT_E_INVALID, "NULL argument");
  if (nsteps < 0) return fail(HIT_E_INVALID, "nsteps must be >= 0");
  int rc;
  if ((rc = check_params(pr))) return rc;
  DeviceGuard dg(p->device);
  return DISPATCH(p, rollout_impl)(p, u_hat, pr, dt, nsteps, out, nullptr, (cudaStream_t)stream);
}

int hit_profile_rollout(hit_plan* p, const void* u_hat, const hit_params* pr, double dt, int64_t nsteps, void* out,
                        double* ms, int* launches, void* stream) {
  if (!p || !u_hat || !out || !ms || !launches) return fail(HIT_E_INVALID, "NULL argument");
  if (nsteps < 1) return fail(HIT_E_INVALID, "nsteps must be >= 1");
  int rc;
  if ((rc = check_params(pr))) return rc;
  DeviceGuard dg(p->device);
  return DISPATCH(p, profile_impl)(p, u_hat, pr, dt, nsteps, out, ms, launches, (cudaStream_t)stream);
}

int hit_rhs_vjp(hit_plan* p, const void* u_hat, const hit_params* pr, double t, const void* ct, void* u_bar,
                double* param_ct, void* stream) {
  (void)t;
  if (!p || !u_hat || !ct || !u_bar) return fail(HIT_E_INVALID, "NULL argument");
  int rc;
  if ((rc = check_params(pr))) return rc;
  DeviceGuard dg(p->device);
  return DISPATCH(p, vjp_entry)(p, 0, u_hat, pr, 0.0, 0, 1, ct, u_bar, param_ct, (cudaStream_t)stream);
}

int hit_rk4_step_vjp(hit_plan* p, const void* u_hat, const hit_params* pr, double dt, double t, const void* ct,
                     void* u_bar, double* param_ct, void* stream) {
  (void)t;
  if (!p || !u_hat || !ct || !u_bar) return fail(HIT_E_INVALID, "NULL argument");
  int rc;
  if ((rc = check_params(pr))) return rc;
  if (pr->flags & HIT_FLAG_INTEGRATING_FACTOR)
    return fail(HIT_E_UNSUPPORTED, "the integrating-factor RK4 step has no transpose");
  DeviceGuard dg(p->device);
  return DISPATCH(p, vjp_entry)(p, 1, u_hat, pr, dt, 1, 1, ct, u_bar, param_ct, (cudaStream_t)stream);
}

int hit_rk4_step_forced_vjp(hit_plan* p, const void* u_hat, const hit_params* pr, const void* f_ext, double dt,
                            double t, const void* ct, void* u_bar, void* f_bar, double* param_ct, void* stream) {
  (void)t;
  if (!p || !u_hat || !f_ext || !ct || !u_bar) return fail(HIT_E_INVALID, "NULL argument");
  int rc;
  if ((rc = check_params(pr))) return rc;
  if (pr->flags & HIT_FLAG_INTEGRATING_FACTOR)
    return fail(HIT_E_UNSUPPORTED, "the integrating-factor RK4 step has no transpose");
  DeviceGuard dg(p->device);
  return DISPATCH(p, forced_vjp_entry)(p, u_hat, pr, f_ext, dt, ct, u_bar, f_bar, param_ct, (cudaStream_t)stream);
}

int hit_axis_fft(hit_plan* p, const void* in, void* out, int ncomp, int axis, int inverse, void* stream) {
  if (!p || !in || !out) return fail(HIT_E_INVALID, "NULL argument");
  if (ncomp < 1 || axis < 0 || axis > 2) return fail(HIT_E_INVALID, "axis_fft: ncomp >= 1, axis in {0, 1, 2}");
  if (axis < 2 && in == out) return fail(HIT_E_INVALID, "axis_fft: in and out must differ");
  DeviceGuard dg(p->device);
  return DISPATCH(p, axis_fft_impl)(p, in, out, ncomp, axis, inverse, (cudaStream_t)stream);
}

int hit_sgs_force_vjp(hit_plan* p, const void* f_bar, void* tau_bar, void* stream) {
  if (!p || !f_bar || !tau_bar) return fail(HIT_E_INVALID, "NULL argument");
  DeviceGuard dg(p->device);
  return DISPATCH(p, sgs_force_vjp_impl)(p, f_bar, tau_bar, (cudaStream_t)stream);
}

int hit_velocity_gradients_vjp(hit_plan* p, const void* grads_bar, void* u_bar, void* stream) {
  if (!p || !grads_bar || !u_bar) return fail(HIT_E_INVALID, "NULL argument");
  DeviceGuard dg(p->device);
  return DISPATCH(p, grad_vjp_impl)(p, grads_bar, u_bar, (cudaStream_t)stream);
}

int hit_rollout_vjp(hit_plan* p, const void* u0, const hit_params* pr, double dt, int64_t nsteps, double t0,
                    int checkpoint_every, const void* ct, void* u0_bar, double* param_ct, void* stream) {
  (void)t0;
  if (!p || !u0 || !ct || !u0_bar) return fail(HIT_E_INVALID, "NULL argument");
  if (nsteps < 0) return fail(HIT_E_INVALID, "nsteps must be >= 0");
  if (checkpoint_every < 1) return fail(HIT_E_INVALID, "checkpoint_every must be >= 1");
  int rc;
  if ((rc = check_params(pr))) return rc;
  if (pr->flags & HIT_FLAG_INTEGRATING_FACTOR)
    return fail(HIT_E_UNSUPPORTED, "the integrating-factor RK4 step has no transpose");
  DeviceGuard dg(p->device);
  const int K = (int)std::min<int64_t>(checkpoint_every, std::max<int64_t>(nsteps, 1));
  return DISPATCH(p, vjp_entry)(p, 2, u0, pr, dt, nsteps, K, ct, u0_bar, param_ct, (cudaStream_t)stream);
}

int hit_velocity_gradients(hit_plan* p, const void* u_hat, void* grads, void* stream) {
  if (!p || !u_hat || !grads) return fail(HIT_E_INVALID, "NULL argument");
  DeviceGuard dg(p->device);
  const Geom g = make_geom(p->Nx, p->Ny, p->Nz, false);
  const size_t es = p->dtype == HIT_DTYPE_F32 ? sizeof(float2) : sizeof(double2);
  int rc;
  if ((rc = ensure(p->ax9, 9 * (size_t)g.Nx * g.Ny * g.Nzh * es))) return rc;
  cudaError_t e = p->dtype == HIT_DTYPE_F32
                      ? launch_grad9<float>(static_cast<const float2*>(u_hat), static_cast<float2*>(p->ax9.p), g,
                                            ktab_of<float>(p), (cudaStream_t)stream)
                      : launch_grad9<double>(static_cast<const double2*>(u_hat), static_cast<double2*>(p->ax9.p), g,
                                             ktab_of<double>(p), (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "velocity_gradients");
  return DISPATCH(p, to_physical_impl)(p, p->ax9.p, 9, grads, (cudaStream_t)stream);
}

namespace {
int sgs_force_entry(hit_plan* p, const void* tau_hat, void* out, void* stream, bool add) {
  if (!p || !tau_hat || !out) return fail(HIT_E_INVALID, "NULL argument");
  DeviceGuard dg(p->device);
  const Geom g = make_geom(p->Nx, p->Ny, p->Nz, false);
  cudaError_t e = p->dtype == HIT_DTYPE_F32
                      ? launch_sgs_force<float>(static_cast<const float2*>(tau_hat), static_cast<float2*>(out), g,
                                                ktab_of<float>(p), (cudaStream_t)stream, add)
                      : launch_sgs_force<double>(static_cast<const double2*>(tau_hat), static_cast<double2*>(out), g,
                                                 ktab_of<double>(p), (cudaStream_t)stream, add);
  if (e != cudaSuccess) return cuda_fail(e, "sgs_force");
  return HIT_OK;
}
}  // namespace

int hit_add_sgs_force(hit_plan* p, const void* tau_hat, void* du, void* stream) {
  return sgs_force_entry(p, tau_hat, du, stream, true);
}

int hit_sgs_force(hit_plan* p, const void* tau_hat, void* f, void* stream) {
  return sgs_force_entry(p, tau_hat, f, stream, false);
}

int hit_tc_gemm_bf16(const void* A, int lda, const void* B, int ldb, float* C, int ldc, int M, int N, int K, int* err,
                     void* stream) {
  if (!A || !B || !C || !err) return fail(HIT_E_INVALID, "NULL argument");
  if (M < 1 || K < 16 || K % 16 || lda % 8 || ldb % 8 || lda < K || ldb < K || ldc < N)
    return fail(HIT_E_INVALID, "tc_gemm: M >= 1, K a multiple of 16, lda/ldb multiples of 8 and >= K, ldc >= N");
  if (N != 16 && N != 32 && N != 64 && N != 128) return fail(HIT_E_INVALID, "tc_gemm: N in {16, 32, 64, 128}");
  if (((uintptr_t)A | (uintptr_t)B) % 16) return fail(HIT_E_INVALID, "tc_gemm: A and B must be 16-byte aligned");
  cudaError_t e = launch_tcgemm(static_cast<const __nv_bfloat16*>(A), lda, static_cast<const __nv_bfloat16*>(B), ldb, C,
                                ldc, M, N, K, err, (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "tc_gemm");
  return HIT_OK;
}

int hit_energy_spectrum(hit_plan* p, const void* u_hat, double* E, double* Ec, void* stream) {
  if (!p || !u_hat) return fail(HIT_E_INVALID, "NULL argument");
  if (!E && !Ec) return fail(HIT_E_INVALID, "no output requested");
  DeviceGuard dg(p->device);
  return DISPATCH(p, diag_impl)(p, u_hat, nullptr, E, Ec, nullptr, (cudaStream_t)stream);
}

int hit_energy_budget(hit_plan* p, const void* u_hat, const hit_params* pr, double* out, void* stream) {
  if (!p || !u_hat || !out) return fail(HIT_E_INVALID, "NULL argument");
  int rc;
  if ((rc = check_params(pr))) return rc;
  DeviceGuard dg(p->device);
  return DISPATCH(p, diag_impl)(p, u_hat, pr, nullptr, nullptr, out, (cudaStream_t)stream);
}

}  // extern "C"
