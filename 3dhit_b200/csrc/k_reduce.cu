// Layout conversion, elementwise spectral operators and the float64
// reductions (spectra, budget, forcing coefficients).
//
// Reductions are two-level and deterministic: each block writes its partial
// sums to a fixed slot, then one finaliser sums the slots in a fixed order
// with Kahan compensation.  Shell indices reproduce the reference's float
// arithmetic exactly: floor(sqrt(k2)/k0 + 0.5) with every operation rounded
// in the run dtype (src/hit3d/diagnostics.py:76-82).
#include "kernels.h"

namespace hit {

template <typename T> __device__ __forceinline__ int shell_of(T k2, T k0);
template <> __device__ __forceinline__ int shell_of<float>(float k2, float k0) {
  return (int)floorf(__fadd_rn(__fdiv_rn(__fsqrt_rn(k2), k0), 0.5f));
}
template <> __device__ __forceinline__ int shell_of<double>(double k2, double k0) {
  return (int)floor(__dadd_rn(__ddiv_rn(__dsqrt_rn(k2), k0), 0.5));
}

// ---------------------------------------------------------------------------
// gather: reference layout -> compact layout (+ optional NSCAL partial sums)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(NT) k_gather(GatherArgs<T> a) {
  __shared__ double red[32];
  const Geom& g = a.g;
  const long long nmodes = (long long)g.Mx * g.My * g.Mzp;
  const long long ce = (long long)g.Nx * g.Ny * g.Nzh;  // ext comp stride
  const long long cc = (long long)g.Mx * g.My * g.Mzp;  // compact comp stride
  double sE = 0, sO = 0, sB = 0;
  for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < nmodes; m += (long long)gridDim.x * NT) {
    const int k = (int)(m % g.Mzp);
    const long long r = m / g.Mzp;
    const int j = (int)(r % g.My), i = (int)(r / g.My);
    V2<T> v[3] = {czero<T>(), czero<T>(), czero<T>()};
    if (k < g.Mz) {
      const int fx = full_pos(i, g.hx, g.Mx, g.Nx), fy = full_pos(j, g.hy, g.My, g.Ny);
      const long long e = ((long long)fx * g.Ny + fy) * g.Nzh + k;
#pragma unroll
      for (int c = 0; c < 3; ++c) v[c] = a.ext[c * ce + e];
      if (a.partial) {
        const T k2 = k2_of(a.k.kx[fx], a.k.ky[fy], a.k.kz[k]);
        double a2 = 0;
#pragma unroll
        for (int c = 0; c < 3; ++c) a2 += (double)v[c].x * v[c].x + (double)v[c].y * v[c].y;
        const double w = herm_weight(g, k);
        sE += w * a2;
        sO += w * (double)k2 * a2;
        if (a.kmin2 <= k2 && k2 <= a.kmax2) sB += w * a2;
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) a.cmp[c * cc + m] = v[c];
  }
  if (a.partial) {
    double r = block_sum_f64(sE, red);
    if (threadIdx.x == 0) a.partial[3 * blockIdx.x + 0] = r;
    r = block_sum_f64(sO, red);
    if (threadIdx.x == 0) a.partial[3 * blockIdx.x + 1] = r;
    r = block_sum_f64(sB, red);
    if (threadIdx.x == 0) a.partial[3 * blockIdx.x + 2] = r;
  }
}

template <typename T> cudaError_t launch_gather(const GatherArgs<T>& a, int nblocks, cudaStream_t st) {
  k_gather<T><<<nblocks, NT, 0, st>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// scatter: compact -> reference layout (modes outside the compact set are 0)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(NT) k_scatter(const V2<T>* __restrict__ cmp, V2<T>* __restrict__ ext, Geom g) {
  const long long nmodes = (long long)g.Nx * g.Ny * g.Nzh;
  const long long cc = (long long)g.Mx * g.My * g.Mzp;
  for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < nmodes; e += (long long)gridDim.x * NT) {
    const int k = (int)(e % g.Nzh);
    const long long r = e / g.Nzh;
    const int fy = (int)(r % g.Ny), fx = (int)(r / g.Ny);
    const int i = compact_row(fx, g.hx, g.Mx, g.Nx), j = compact_row(fy, g.hy, g.My, g.Ny);
    const bool kept = i >= 0 && j >= 0 && k < g.Mz;
    const long long m = kept ? ((long long)i * g.My + j) * g.Mzp + k : 0;
#pragma unroll
    for (int c = 0; c < 3; ++c) ext[c * nmodes + e] = kept ? cmp[c * cc + m] : czero<T>();
  }
}

static int grid_for(long long n) {
  long long b = (n + NT - 1) / NT;
  return (int)(b < 8 * 148 ? (b < 1 ? 1 : b) : 8 * 148);
}

template <typename T> cudaError_t launch_scatter(const V2<T>* cmp, V2<T>* ext, const Geom& g, cudaStream_t st) {
  k_scatter<T><<<grid_for((long long)g.Nx * g.Ny * g.Nzh), NT, 0, st>>>(cmp, ext, g);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// flag modes outside the 2/3 box that are nonzero
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(NT) k_check_box(const V2<T>* __restrict__ ext, Geom g, int* flag) {
  const long long nmodes = (long long)g.Nx * g.Ny * g.Nzh;
  int found = 0;
  for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < nmodes; e += (long long)gridDim.x * NT) {
    const int k = (int)(e % g.Nzh);
    const long long r = e / g.Nzh;
    const int fy = (int)(r % g.Ny), fx = (int)(r / g.Ny);
    const bool in_box = abs(freq_of(fx, g.Nx)) <= g.cx && abs(freq_of(fy, g.Ny)) <= g.cy && k <= g.cz;
    if (!in_box) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const V2<T> v = ext[c * nmodes + e];
        found |= (v.x != T(0) || v.y != T(0));  // NaN compares unequal -> flagged
      }
    }
  }
  if (__syncthreads_or(found) && threadIdx.x == 0) atomicOr(flag, 1);
}

template <typename T> cudaError_t launch_check_box(const V2<T>* ext, const Geom& g, int* flag, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(flag, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  k_check_box<T><<<grid_for((long long)g.Nx * g.Ny * g.Nzh), NT, 0, st>>>(ext, g, flag);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// project(dealias(u)) in the reference layout (src/hit3d/grid.py:166-178)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(NT) k_dealias_project(const V2<T>* __restrict__ in, V2<T>* __restrict__ out, Geom g,
                                                        KTab<T> kt, int dd, int pp) {
  const long long nmodes = (long long)g.Nx * g.Ny * g.Nzh;
  for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < nmodes; e += (long long)gridDim.x * NT) {
    const int k = (int)(e % g.Nzh);
    const long long r = e / g.Nzh;
    const int fy = (int)(r % g.Ny), fx = (int)(r / g.Ny);
    V2<T> u[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) u[c] = in[c * nmodes + e];
    if (dd && !in_dealias(g, fx, fy, k)) u[0] = u[1] = u[2] = czero<T>();
    if (pp) {
      const T kx = kt.kx[fx], ky = kt.ky[fy], kz = kt.kz[k];
      const T ik2 = inv_k2_of(k2_of(kx, ky, kz));
      V2<T> div;
      div.x = (kx * u[0].x + ky * u[1].x + kz * u[2].x) * ik2;
      div.y = (kx * u[0].y + ky * u[1].y + kz * u[2].y) * ik2;
      u[0] = csub(u[0], cscale(div, kx));
      u[1] = csub(u[1], cscale(div, ky));
      u[2] = csub(u[2], cscale(div, kz));
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c * nmodes + e] = u[c];
  }
}

template <typename T>
cudaError_t launch_dealias_project(const V2<T>* in, V2<T>* out, const Geom& g, KTab<T> k, int dd, int pp, cudaStream_t st) {
  k_dealias_project<T><<<grid_for((long long)g.Nx * g.Ny * g.Nzh), NT, 0, st>>>(in, out, g, k, dd, pp);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// per-block spectral sums: shells (per component) and NSCAL scalars,
// compensated and in a fixed order (bit-identical from run to run)
// ---------------------------------------------------------------------------
struct KahanAcc {  // compensated running sum
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double x) {
    const double y = x - c;
    const double t = s + y;
    c = (t - s) - y;
    s = t;
  }
  __device__ __forceinline__ double value() const { return s - c; }
};

constexpr int MS_WARPS = 4;  // warps per k_mode_sums block

// A warp takes 32 consecutive kz modes of one (kx, ky) row at a time (the
// chunks are dealt to the warps of the grid in a fixed order).  Along a row
// |k| and hence the shell index never decrease with kz, so the lanes of one
// shell form contiguous runs: a segmented shuffle scan in lane order gives
// each run's sum in its last lane, which adds it (Kahan) to the warp's own
// bins in shared memory; different runs have different shells, so no two
// lanes touch one bin.  E, Omega and the band energy are per-lane Kahan sums.
// At the end the warps' bins are added in warp order and the scalars by a
// fixed shuffle tree, so the result does not depend on scheduling.
template <typename T>
__global__ void __launch_bounds__(MS_WARPS * 32) k_mode_sums(ModeSumArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nb3 = 3 * a.nshell;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* bs = reinterpret_cast<double*>(smem_raw);  // [warp][nb3] sums, then [warp][nb3] compensations
  double* bc = bs + MS_WARPS * nb3;
  __shared__ double red[32];
  for (int e = threadIdx.x; e < 2 * MS_WARPS * nb3; e += MS_WARPS * 32) bs[e] = 0.0;
  __syncthreads();
  const Geom& g = a.g;
  const int nck = (g.Mz + 31) / 32;
  const long long nchunks = (long long)g.Mx * g.My * nck;
  double* wb = bs + warp * nb3;
  double* wc = bc + warp * nb3;
  KahanAcc sE, sO, sB;
  for (long long ch = (long long)blockIdx.x * MS_WARPS + warp; ch < nchunks; ch += (long long)gridDim.x * MS_WARPS) {
    const long long row = ch / nck;
    const int k = (int)(ch % nck) * 32 + lane;
    const int j = (int)(row % g.My), i = (int)(row / g.My);
    const bool on = k < g.Mz;
    const int fx = full_pos(i, g.hx, g.Mx, g.Nx), fy = full_pos(j, g.hy, g.My, g.Ny);
    double e[3] = {0.0, 0.0, 0.0};
    int s = 0x7fffffff;  // lanes past the row: a key no real shell has
    if (on) {
      const long long off = (long long)i * a.c_x + (long long)j * a.c_y + k;
      const T k2 = k2_of(a.k.kx[fx], a.k.ky[fy], a.k.kz[k]);
      const double w = herm_weight(g, k);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const V2<T> v = a.u[c * a.c_c + off];
        e[c] = w * ((double)v.x * v.x + (double)v.y * v.y);
      }
      const double t = (e[0] + e[1]) + e[2];
      sE.add(t);
      sO.add((double)k2 * t);
      if (a.kmin2 <= k2 && k2 <= a.kmax2) sB.add(t);
      if (a.nshell > 0) {
        s = shell_of<T>(k2, a.k0);
        if (s < 0 || s >= a.nshell) s = 0x7ffffffe;  // not binned (a key of its own)
      }
    }
    if (a.nshell > 0) {
      // segmented inclusive scan over runs of equal s (contiguous in lane order)
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int so = __shfl_up_sync(0xffffffffu, s, d);
        double up[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) up[c] = __shfl_up_sync(0xffffffffu, e[c], d);
        if (lane >= d && so == s) {
#pragma unroll
          for (int c = 0; c < 3; ++c) e[c] += up[c];
        }
      }
      const int sn = __shfl_down_sync(0xffffffffu, s, 1);
      if (on && s < a.nshell && (lane == 31 || sn != s)) {  // last lane of its run
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const int b = c * a.nshell + s;
          const double y = e[c] - wc[b];
          const double t = wb[b] + y;
          wc[b] = (t - wb[b]) - y;
          wb[b] = t;
        }
      }
      __syncwarp();
    }
  }
  const int NV = nb3 + NSCAL;
  double* out = a.partial + (long long)blockIdx.x * NV;
  double r = block_sum_f64(sE.value(), red);
  if (threadIdx.x == 0) out[nb3 + 0] = r;
  r = block_sum_f64(sO.value(), red);
  if (threadIdx.x == 0) out[nb3 + 1] = r;
  r = block_sum_f64(sB.value(), red);
  if (threadIdx.x == 0) out[nb3 + 2] = r;
  __syncthreads();
  for (int b = threadIdx.x; b < nb3; b += MS_WARPS * 32) {
    KahanAcc t;
#pragma unroll
    for (int w = 0; w < MS_WARPS; ++w) t.add(bs[w * nb3 + b] - bc[w * nb3 + b]);
    out[b] = t.value();
  }
}

template <typename T> size_t mode_sums_smem(int nshell) {
  return sizeof(double) * 2 * MS_WARPS * 3 * (size_t)(nshell > 0 ? nshell : 1);
}

template <typename T> cudaError_t launch_mode_sums(const ModeSumArgs<T>& a, int nblocks, cudaStream_t st) {
  const size_t smem = mode_sums_smem<T>(a.nshell);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k_mode_sums<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_mode_sums<T><<<nblocks, MS_WARPS * 32, smem, st>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// out = u * c[shell(k)] (random_field's per-shell rescale, src/hit3d/fields.py:51-68)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(NT) k_shell_scale(const V2<T>* __restrict__ in, V2<T>* __restrict__ out, Geom g,
                                                    KTab<T> kt, T k0, const double* __restrict__ c, int smax) {
  const long long nmodes = (long long)g.Nx * g.Ny * g.Nzh;
  for (long long e = blockIdx.x * (long long)NT + threadIdx.x; e < nmodes; e += (long long)gridDim.x * NT) {
    const int k = (int)(e % g.Nzh);
    const long long r = e / g.Nzh;
    const int fy = (int)(r % g.Ny), fx = (int)(r / g.Ny);
    int s = shell_of<T>(k2_of(kt.kx[fx], kt.ky[fy], kt.kz[k]), k0);
    s = s < 0 ? 0 : (s > smax ? smax : s);  // out-of-range gathers clamp, as jnp indexing does
    const T f = (T)c[s];
#pragma unroll
    for (int q = 0; q < 3; ++q) out[q * nmodes + e] = cscale(in[q * nmodes + e], f);
  }
}

template <typename T>
cudaError_t launch_shell_scale(const V2<T>* in, V2<T>* out, const Geom& g, KTab<T> k, T k0, const double* c, int smax,
                               cudaStream_t st) {
  k_shell_scale<T><<<grid_for((long long)g.Nx * g.Ny * g.Nzh), NT, 0, st>>>(in, out, g, k, k0, c, smax);
  return cudaGetLastError();
}
template cudaError_t launch_shell_scale<float>(const float2*, float2*, const Geom&, KTab<float>, float, const double*, int, cudaStream_t);
template cudaError_t launch_shell_scale<double>(const double2*, double2*, const Geom&, KTab<double>, double, const double*, int, cudaStream_t);

// ---------------------------------------------------------------------------
// finalisers
// ---------------------------------------------------------------------------
struct Kahan {
  double s = 0.0, c = 0.0;
  __device__ void add(double x) {
    const double y = x - c;
    const double t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

// Deterministic block-wide Kahan sum of column v of partial[nb][stride].
__device__ double kahan_column(const double* partial, int nb, int stride, int v, double* red) {
  Kahan k;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) k.add(partial[(long long)b * stride + v]);
  return block_sum_f64(k.s - k.c, red);
}

__device__ __forceinline__ double forcing_coef(int forcing, double E, double Om, double twoEb, double nu, double eps,
                                               double Et, double tau, double tiny, double A) {
  if (forcing == 1) return A;
  if (forcing == 2) return twoEb > tiny ? eps / twoEb : 0.0;
  if (forcing == 3) {
    const double relax = (tau > 0.0 && isfinite(tau)) ? (E - Et) / tau : 0.0;
    return E > 0.0 ? (2.0 * nu * Om - relax) / (2.0 * E) : 0.0;
  }
  return 0.0;
}

// One 1024-thread block: thread t Kahan-sums rows t, t + 1024, ... of the
// three columns in order, issuing the loads of CB rows before adding them (the
// row chain is latency-bound otherwise), then fixed shuffle trees combine the
// threads.
constexpr int COEF_THREADS = 1024;
__global__ void __launch_bounds__(COEF_THREADS) k_finalize_coef(CoefArgs a) {
  __shared__ double red[96];
  pdl_wait();
  pdl_trigger();
  constexpr int CB = 4;
  Kahan k0, k1, k2;
  for (int b0 = threadIdx.x; b0 < a.nblocks; b0 += CB * COEF_THREADS) {
    double v[CB][3];
#pragma unroll
    for (int i = 0; i < CB; ++i) {
      const int b = b0 + i * COEF_THREADS;
#pragma unroll
      for (int c = 0; c < 3; ++c) v[i][c] = b < a.nblocks ? a.partial[3 * (long long)b + c] : 0.0;
    }
#pragma unroll
    for (int i = 0; i < CB; ++i) {
      if (b0 + i * COEF_THREADS < a.nblocks) {
        k0.add(v[i][0]);
        k1.add(v[i][1]);
        k2.add(v[i][2]);
      }
    }
  }
  double S0 = k0.s - k0.c, S1 = k1.s - k1.c, S2 = k2.s - k2.c;
  block_sum3_f64(S0, S1, S2, red);
  if (threadIdx.x == 0) {
    const double E = S0 / (2.0 * a.ntot2), Om = S1 / (2.0 * a.ntot2), twoEb = S2 / a.ntot2;
    a.coef[0] = forcing_coef(a.forcing, E, Om, twoEb, a.nu, a.eps, a.E_target, a.tau, a.tiny, 0.0);
    a.coef[1] = E;
    a.coef[2] = Om;
    a.coef[3] = twoEb;
  }
}

cudaError_t launch_finalize_coef(const CoefArgs& a, cudaStream_t st) {
  return launch_pdl(k_finalize_coef, 1, COEF_THREADS, 0, st, a);
}

__global__ void k_finalize_sums(SumArgs a) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= a.nvals) return;
  Kahan k;
  for (int b = 0; b < a.nblocks; ++b) k.add(a.partial[(long long)b * a.nvals + v]);
  a.sums[v] = k.s - k.c;
}

cudaError_t launch_finalize_sums(const SumArgs& a, cudaStream_t st) {
  k_finalize_sums<<<(a.nvals + NT - 1) / NT, NT, 0, st>>>(a);
  return cudaGetLastError();
}

__global__ void k_finalize_budget(BudgetArgs a) {
  const int ns = a.nshell;
  const double inv = 1.0 / (2.0 * a.ntot2);
  for (int s = 1 + threadIdx.x; s < ns; s += blockDim.x) {
    const double c0 = a.sums[s] * inv, c1 = a.sums[ns + s] * inv, c2 = a.sums[2 * ns + s] * inv;
    if (a.spec) a.spec[s - 1] = c0 + c1 + c2;
    if (a.comp) {
      a.comp[s - 1] = c0;
      a.comp[(ns - 1) + s - 1] = c1;
      a.comp[2 * (ns - 1) + s - 1] = c2;
    }
  }
  if (threadIdx.x == 0 && a.budget) {
    const double* sc = a.sums + 3 * ns;
    const double E = sc[0] * inv, Om = sc[1] * inv, twoEb = sc[2] / a.ntot2;
    const double cf = forcing_coef(a.forcing, E, Om, twoEb, a.nu, a.eps, a.E_target, a.tau, a.tiny, a.A);
    double P = 0.0;
    if (a.forcing == 1 || a.forcing == 3) P = cf * 2.0 * E;
    else if (a.forcing == 2) P = twoEb > a.tiny ? a.eps : 0.0;
    a.budget[0] = E;
    a.budget[1] = 2.0 * a.nu * Om;
    a.budget[2] = P;
    a.budget[3] = Om;
  }
}

cudaError_t launch_finalize_budget(const BudgetArgs& a, cudaStream_t st) {
  k_finalize_budget<<<1, NT, 0, st>>>(a);
  return cudaGetLastError();
}

template cudaError_t launch_gather<float>(const GatherArgs<float>&, int, cudaStream_t);
template cudaError_t launch_gather<double>(const GatherArgs<double>&, int, cudaStream_t);
template cudaError_t launch_scatter<float>(const float2*, float2*, const Geom&, cudaStream_t);
template cudaError_t launch_scatter<double>(const double2*, double2*, const Geom&, cudaStream_t);
template cudaError_t launch_check_box<float>(const float2*, const Geom&, int*, cudaStream_t);
template cudaError_t launch_check_box<double>(const double2*, const Geom&, int*, cudaStream_t);
template cudaError_t launch_dealias_project<float>(const float2*, float2*, const Geom&, KTab<float>, int, int, cudaStream_t);
template cudaError_t launch_dealias_project<double>(const double2*, double2*, const Geom&, KTab<double>, int, int, cudaStream_t);
template cudaError_t launch_mode_sums<float>(const ModeSumArgs<float>&, int, cudaStream_t);
template cudaError_t launch_mode_sums<double>(const ModeSumArgs<double>&, int, cudaStream_t);

}  // namespace hit
