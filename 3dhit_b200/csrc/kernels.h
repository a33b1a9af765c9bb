// Argument blocks and host launchers of the HIT3D kernels (internal header;
// the public boundary is include/hit3d.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <utility>

#include <cuda_bf16.h>

#include "common.cuh"

namespace hit {

// Launch with programmatic stream serialization (see pdl_wait).
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), int grid, int block, size_t smem, cudaStream_t st, Args&&... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

constexpr int NT = 256;   // threads per block of the axis, z and reduction kernels
constexpr int NTP = 512;  // threads per block of k_p1/k_p3 (one 131 KB CTA per SM)

// Columns (contiguous z entries) per x/y tile: one tile column block is at
// most 32 KB, so P1/P3 (four tiles) fit in 128 KB of shared memory.
template <typename T> __host__ __device__ constexpr int tile_w(int N) {
  return (32768 / (N * (int)sizeof(V2<T>))) >= 8 ? 8 : (32768 / (N * (int)sizeof(V2<T>)));
}
// k_p1/k_p3 tile width (same as the axis kernels).
template <typename T> __host__ __device__ constexpr int tile_wp(int N) { return tile_w<T>(N); }

// Plain column FFT along a strided axis ("a") of a 4-D array indexed
// (comp, a, o, z): element at src + c*s_c + a*s_a + o*s_o + z.  Input rows
// along a are compact (Min stored rows, hin non-negative), output rows compact
// (Mout, hout); nz valid z columns.  grid = (ceil(nz/W), n_o, ncomp).
template <typename T> struct AxisArgs {
  const V2<T>* src;
  V2<T>* dst;
  long long s_c, s_a, s_o;
  long long d_c, d_a, d_o;
  int Min, hin, Mout, hout;
  int nz;
  const V2<T>* tw;
  int src_cols;  // entries per source row that may be read (0: nz); staging reads whole W-column tiles
  int br, ka, kb, pb;  // TMA staging (set by the launcher): box rows, boxes per half, rows of the second half
};

// P1: x-inverse of the stage input and of curl(u): 3 compact components in,
// 6 x-physical components out (u_x,u_y,u_z, w_x,w_y,w_z).  grid = (Mzp/W, My).
template <typename T> struct P1Args {
  const V2<T>* s;   // (3, Mx, My, Mzp)
  long long s_c, s_x;
  int les;          // 1: 12 outputs, u and the velocity gradients (see p1les_body)
  V2<T>* t6;        // (6, Nx, My, Mzp)
  long long t_c, t_x;
  Geom g;
  KTab<T> k;
  const V2<T>* tw;
};

// P3: x-forward of the nonlinear term, RHS epilogue (forcing, dealias,
// projection, viscous term), RK4 stage update, optional fused P1 of the new
// stage input, optional per-block partial sums of the new stage input.
template <typename T> struct P3Args {
  const V2<T>* t3;  // (3, Nx, My, Mzp)
  long long t_c, t_x;
  V2<T>* u;         // state (3, Mx, My, Mzp)
  V2<T>* acc;       // RK accumulator
  V2<T>* s;         // stage input of stages 2..4
  V2<T>* out;       // stage 0: du output
  long long c_c, c_x;
  V2<T>* t6;        // fused P1 output
  long long t6_c, t6_x;
  Geom g;
  KTab<T> k;
  const V2<T>* tw;
  int stage;        // 0: rhs only (u_stage = u); 1..4: RK4 stage
  int fuse_p1;
  int ifrk;         // 1: integrating-factor RK4 stages (nu = 0 here, the
                    //    viscous operator enters through e^{-nu k^2 dt/2})
  T nu, a_next, dt6;
  T nuh;            // nu dt / 2 (integrating-factor RK4)
  int forcing;
  T fA, kmin2, kmax2;
  const double* coef;  // coef[0]: band c or hold-energy A (float64)
  double* partial;     // per-block (3 per block) sums of the new stage input
  const V2<T>* fext;   // optional external force (compact layout, index o like u),
                       // added to the nonlinear term before the mask and projection
  // fused LES stage (shared-memory mode only): t3 holds 9 x-physical fields,
  // u x w then the SGS stress tau (xx, yy, zz, xy, xz, yz); the epilogue forms
  // f = -i k_j tau_hat_ij, adds it to the nonlinear term and stores it at
  // fext_out (compact layout) for the step's later stages
  int les;
  V2<T>* fext_out;
};

// Fused z pass of the RHS: per (x, y) row, c2r of 6 components, u x w,
// r2c of 3 components, in place (output = first 3 components).
template <typename T> struct ZCrossArgs {
  V2<T>* buf;  // (6, Nx, Ny, Mzp)
  long long c_stride;
  int nrows, Mz, Mzp;
  T scale;     // 1/(Nx Ny Nz)
  const V2<T>* tw;
};

// z pass of the fused LES stage (k_zles, float32): per (x, y) row, c2r of u
// and the nine velocity gradients, u x w and the closure MLP per physical
// point, r2c of the three products and the six SGS stresses (xx, yy, zz,
// xy, xz, yz), written over the first nine of the twelve input rows.
struct ZLesArgs {
  float2* buf;  // (12, Nx, Ny, Mzp)
  long long c_stride;
  int nrows, Mz, Mzp;
  float scale;  // 1/(Nx Ny Nz)
  const float2* tw;
  const __nv_bfloat16 *w1t, *w2t, *w3t, *w4t;  // the MLP's forward weights (hit_mlp_weights)
  const float *b2, *b3, *b4;
  int* err;     // set when an MMA completion wait gave up
};
cudaError_t launch_zles(int H, const ZLesArgs& a, cudaStream_t st);
bool zles_supported(int Nz);

// Plain z c2r / r2c for to_physical / to_spectral.
template <typename T> struct ZRealArgs {
  V2<T>* cbuf;        // complex rows, stride Mzp, Mz = Nz/2+1 valid
  T* rbuf;            // real rows, stride Nz
  long long cc_stride, rc_stride;  // per-component strides
  int nrows, Mz, Mzp;
  T scale;
  const V2<T>* tw;
};

// One int per device ordinal, 0 until set.  Kernel attributes (the dynamic
// shared-memory opt-in, the carveout), occupancy and SM counts belong to one
// device's context, so launchers keep their one-time set-up and cached launch
// sizes per device.  The slots are atomic: host threads launching on the same
// device may both run the first set-up, which is idempotent.  Devices past
// kMaxDevices get no slot and redo the set-up on every launch.
constexpr int kMaxDevices = 64;
struct PerDevice {
  std::atomic<int> v[kMaxDevices];
  PerDevice() {
    for (auto& x : v) x.store(0, std::memory_order_relaxed);
  }
  std::atomic<int>* here() {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDevices) return nullptr;
    return &v[d];
  }
};

// Runs f() (returning cudaError_t) once per device; a failed f is retried on
// the next call.
template <typename F> cudaError_t once_per_device(PerDevice& done, F&& f) {
  std::atomic<int>* s = done.here();
  if (s && s->load(std::memory_order_acquire)) return cudaSuccess;
  const cudaError_t e = f();
  if (e == cudaSuccess && s) s->store(1, std::memory_order_release);
  return e;
}

// Persistent launch size: the number of blocks that stay resident (the FFT
// kernels loop over their tiles, filling their shared twiddle tables once),
// cached per device.
template <typename K> int resident_grid(K kernel, int threads, size_t smem, long long ntiles, PerDevice& cache) {
  std::atomic<int>* slot = cache.here();
  int n = slot ? slot->load(std::memory_order_relaxed) : 0;
  if (n == 0) {
    int dev = 0, sms = 0, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem);
    n = (occ > 0 ? occ : 1) * (sms > 0 ? sms : 1);
    if (slot) slot->store(n, std::memory_order_relaxed);
  }
  return (int)(ntiles < n ? (ntiles > 0 ? ntiles : 1) : n);
}

// Launchers (return cudaError_t of the launch).
template <typename T> cudaError_t launch_axis(int N, bool inv, const AxisArgs<T>& a, int nzt, int no, int nc, cudaStream_t st);
template <typename T> cudaError_t launch_p1(const P1Args<T>& a, cudaStream_t st);
template <typename T> cudaError_t launch_p3(const P3Args<T>& a, cudaStream_t st);
template <typename T> cudaError_t launch_zcross(int H, const ZCrossArgs<T>& a, cudaStream_t st);
template <typename T> cudaError_t launch_zc2r(int H, const ZRealArgs<T>& a, int ncomp, cudaStream_t st);
template <typename T> cudaError_t launch_zr2c(int H, const ZRealArgs<T>& a, int ncomp, cudaStream_t st);
template <typename T> cudaError_t prepare_fft_kernels(int Nx, int Ny, int Nz);
template <typename T> cudaError_t prepare_axis_kernels(int Nx);
int p3_num_blocks(const Geom& g, int W);
template <typename T> int p3_tile_w(int Nx);
cudaError_t take_axis_timeout(int* flag);
cudaError_t take_z_timeout(int* flag);
cudaError_t set_axis_wait_limit(int polls);
cudaError_t set_z_wait_limit(int polls);
template <typename T> int axis_tile_w(int N);

// ---- reductions / elementwise (k_reduce.cu) ----------------------------------
// Scalar sums over modes: index 0: sum w|u|^2, 1: sum w k2 |u|^2, 2: band sum w|u|^2
constexpr int NSCAL = 3;

template <typename T> struct ModeSumArgs {
  const V2<T>* u;        // 3 components
  long long c_c, c_x, c_y;  // strides (comp, x-row, y-row)
  Geom g;                // compact layout of u
  KTab<T> k;
  T kmin2, kmax2;        // band limits (squared, in the run dtype)
  T k0;                  // shell width 2 pi / Lx in the run dtype
  int nshell;            // smax + 1 bins (0 = no spectrum)
  double* partial;       // [nblocks][3*nshell + NSCAL]
};

template <typename T> struct GatherArgs {
  const V2<T>* ext;   // (3, Nx, Ny, Nzh)
  V2<T>* cmp;         // (3, Mx, My, Mzp)
  Geom g;
  KTab<T> k;
  T kmin2, kmax2;
  double* partial;    // nullable: per-block NSCAL sums of the gathered state
};

template <typename T> cudaError_t launch_gather(const GatherArgs<T>& a, int nblocks, cudaStream_t st);
template <typename T> cudaError_t launch_scatter(const V2<T>* cmp, V2<T>* ext, const Geom& g, cudaStream_t st);
template <typename T> cudaError_t launch_check_box(const V2<T>* ext, const Geom& g, int* flag, cudaStream_t st);
template <typename T> cudaError_t launch_dealias_project(const V2<T>* in, V2<T>* out, const Geom& g, KTab<T> k, int dd, int pp, cudaStream_t st);
template <typename T> cudaError_t launch_mode_sums(const ModeSumArgs<T>& a, int nblocks, cudaStream_t st);
template <typename T> cudaError_t launch_shell_scale(const V2<T>* in, V2<T>* out, const Geom& g, KTab<T> k, T k0, const double* c, int smax, cudaStream_t st);

// Finalisers (deterministic, one pass over the per-block partials).
struct CoefArgs {
  const double* partial;
  int nblocks;
  int forcing;
  double ntot2, nu, eps, E_target, tau, tiny;
  double* coef;  // coef[0] = forcing coefficient, coef[1..3] = raw sums
};
cudaError_t launch_finalize_coef(const CoefArgs& a, cudaStream_t st);

// Discrete adjoint of the RHS (k_adjoint.cu), reference layout.
template <typename T> struct AdjArgs {
  const V2<T>* u;   // state (3, Nx, Ny, Nzh)
  const V2<T>* v;   // cotangent of rhs(u)
  V2<T>* x9;        // transform inputs [u, 1j k x u, pv / w] (9 components)
  const V2<T>* s6;  // rfftn(om x g), rfftn(g x u) (6 components)
  V2<T>* ub;        // cotangent of u (output)
  const double* scal;
  double* partial;  // 6 per block
  Geom g;
  KTab<T> k;
  T nu, kmin2, kmax2;
};
struct AdjCoefArgs {
  const double* sums;  // the 6 finalised sums
  double* scal;        // 5 scalars for k_adj_prep
  double* pct;         // parameter cotangents (nu, A, eps), added to
  int forcing;
  double ntot2, nu, A, eps, E_target, tau, tiny;
};
template <typename T> cudaError_t launch_adj_sums(const AdjArgs<T>& a, int nblocks, cudaStream_t st);
cudaError_t launch_adj_coef(const AdjCoefArgs& a, cudaStream_t st);
template <typename T> cudaError_t launch_adj_prep(const AdjArgs<T>& a, cudaStream_t st);
template <typename T> cudaError_t launch_adj_cross(T* p, long long n, cudaStream_t st);
template <typename T> cudaError_t launch_adj_combine(const AdjArgs<T>& a, cudaStream_t st);
template <typename T>
cudaError_t launch_axpby(const V2<T>* x, T alpha, const V2<T>* y, T beta, V2<T>* out, long long n, cudaStream_t st);
template <typename T> cudaError_t launch_grad9(const V2<T>* u, V2<T>* g, const Geom& gm, KTab<T> kt, cudaStream_t st);
template <typename T>
cudaError_t launch_sgs_force(const V2<T>* t, V2<T>* du, const Geom& gm, KTab<T> kt, cudaStream_t st, bool add);
template <typename T>
cudaError_t launch_sgs_force_vjp(const V2<T>* fb, V2<T>* tb, const Geom& gm, KTab<T> kt, T scale, cudaStream_t st);
template <typename T>
cudaError_t launch_grad9_vjp(const V2<T>* G, V2<T>* ub, const Geom& gm, KTab<T> kt, T inv_n3, cudaStream_t st);

cudaError_t launch_tcgemm(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, float* C, int ldc, int M,
                          int N, int K, int* err, cudaStream_t st, int splits = 1, float* work = nullptr);

// Learned-closure MLP (k_mlp.cu).  Weights bf16 row-major: forward W^T of
// layers 1-4 ([64][16], [64][64], [64][64], [16][64]; W1 row 15 of the input
// holds b1) and backward W of layers 2-4 ([64][64], [64][64], [64][16]).
struct MlpArgs {
  const __nv_bfloat16 *w1t, *w2t, *w3t, *w4t, *w2, *w3, *w4;
  const float *b2, *b3, *b4;
  const float* x;    // feature f of point p at x[f * x_sf + p * x_sp]
  const float* tau;  // [P][6] targets (NULL: inference only)
  float* y;          // output c of point p at y[c * y_sf + p * y_sp] (may be NULL when training)
  long long P, x_sf, x_sp, y_sf, y_sp;
  float inv_count;   // 1 / (P * 6)
  __nv_bfloat16 *aT0, *aT1, *aT2, *aT3;     // [16|65][P] activations (+ ones row)
  __nv_bfloat16 *dzT1, *dzT2, *dzT3, *dzT4;  // [64|64|64|16][P]
  double* loss;      // [grid] partial sums of (y - tau)^2
  int* err;
  // vector-Jacobian mode (training instantiation): with ybar set, dL/dy of
  // point p, component c is ybar[c * yb_sf + p * yb_sp] (instead of the MSE
  // gradient of tau); with xbar set (and w1, the backward layer-1 weight W1
  // [16][64], rows 0-8 used), dL/dx of feature f goes to xbar[f * x_sf + p * x_sp]
  const float* ybar;
  long long yb_sf, yb_sp;
  float* xbar;
  const __nv_bfloat16* w1;
};
size_t mlp_smem_bytes();
cudaError_t launch_mlp(const MlpArgs& a, int grid, cudaStream_t st);

struct SumArgs {
  const double* partial;
  int nblocks, nvals;
  double* sums;  // [nvals], Kahan-compensated block sums
};
cudaError_t launch_finalize_sums(const SumArgs& a, cudaStream_t st);

struct BudgetArgs {
  const double* sums;  // [3*nshell + NSCAL]
  int nshell;
  double* spec;        // nullable [nshell-1]   (shells 1..smax)
  double* comp;        // nullable [3*(nshell-1)]
  double* budget;      // nullable [4]: E, eps, P, Omega
  int forcing;
  double ntot2, nu, A, eps, E_target, tau, tiny;
};
cudaError_t launch_finalize_budget(const BudgetArgs& a, cudaStream_t st);

}  // namespace hit
