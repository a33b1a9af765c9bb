// Pointwise and reduction kernels of the discrete adjoint (vector-Jacobian
// product) of the RHS, over the reference layout (3, Nx, Ny, Nz/2+1).
//
// The reference differentiates rhs (src/hit3d/navierstokes.py:62-97) with
// jax.vjp; this is its transpose written out.  A cotangent is dL/dRe +
// i dL/dIm of the stored half-spectrum entries (inner product
// sum Re(conj(a) b) over the stored array).  With pv = project(dealias(v))
// (both self-adjoint), w the Hermitian weights (1 on kz = 0 and the Nyquist
// plane, 2 elsewhere), u = irfftn(u_hat), om = irfftn(1j k x u_hat) and
// g = irfftn(pv / w), the cotangent of u_hat is
//   -nu k2 v                                    (viscous term)
//   + forcing'(u_hat)^T pv                      (forcing term, forcing.py)
//   + w (rfftn(om x g) + 1j k x rfftn(g x u))   (u x w: the transposes of
//                                                irfftn and rfftn are
//                                                w rfftn / N^3 and
//                                                N^3 irfftn(. / w)).
// Forcing coefficients that depend on u_hat (band: eps / 2E_band, hold
// energy: (2 nu Omega - (E - E_target)/tau) / 2E) add their chain-rule terms;
// the float64 sums they need come from k_adj_sums.
#include "kernels.h"

namespace hit {

namespace {
int grid_of(long long n) { return (int)std::min<long long>((n + NT - 1) / NT, 16 * 148); }

template <typename T> struct Mode {
  T kx, ky, kz, k2, ik2;
  int w;       // Hermitian weight
  bool keep;   // inside the 2/3 box (dealias mask)
};

template <typename T>
__device__ __forceinline__ Mode<T> mode_of(long long m, const Geom& g, const KTab<T>& kt, int& fx, int& fy, int& z) {
  z = (int)(m % g.Nzh);
  const long long r = m / g.Nzh;
  fy = (int)(r % g.Ny);
  fx = (int)(r / g.Ny);
  Mode<T> d;
  d.kx = kt.kx[fx];
  d.ky = kt.ky[fy];
  d.kz = kt.kz[z];
  d.k2 = k2_of(d.kx, d.ky, d.kz);
  d.ik2 = inv_k2_of(d.k2);
  d.w = herm_weight(g, z);
  d.keep = in_dealias(g, fx, fy, z);
  return d;
}

// project(dealias(v)) of one mode, in the reference's operation order
// (src/hit3d/grid.py:166-178)
template <typename T> __device__ __forceinline__ void proj_mask(const Mode<T>& d, V2<T> (&v)[3]) {
  if (!d.keep) {
    v[0] = v[1] = v[2] = czero<T>();
    return;
  }
  V2<T> div;
  div.x = (d.kx * v[0].x + d.ky * v[1].x + d.kz * v[2].x) * d.ik2;
  div.y = (d.kx * v[0].y + d.ky * v[1].y + d.kz * v[2].y) * d.ik2;
  v[0] = csub(v[0], cscale(div, d.kx));
  v[1] = csub(v[1], cscale(div, d.ky));
  v[2] = csub(v[2], cscale(div, d.kz));
}

template <typename T> __device__ __forceinline__ double re_dot3(const V2<T> (&a)[3], const V2<T> (&b)[3]) {
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < 3; ++c) s += (double)a[c].x * b[c].x + (double)a[c].y * b[c].y;
  return s;
}

// 1j k x a
template <typename T> __device__ __forceinline__ void curl_of(const Mode<T>& d, const V2<T> (&a)[3], V2<T> (&o)[3]) {
  V2<T> t[3];
  t[0].x = d.ky * a[2].x - d.kz * a[1].x;
  t[0].y = d.ky * a[2].y - d.kz * a[1].y;
  t[1].x = d.kz * a[0].x - d.kx * a[2].x;
  t[1].y = d.kz * a[0].y - d.kx * a[2].y;
  t[2].x = d.kx * a[1].x - d.ky * a[0].x;
  t[2].y = d.kx * a[1].y - d.ky * a[0].y;
#pragma unroll
  for (int c = 0; c < 3; ++c) o[c] = cmul_i(t[c]);
}
}  // namespace

// Per-block float64 partial sums (6 per block):
//   0: sum Re(conj(pv) u)          1: the same over the band
//   2: sum k2 Re(conj(v) u)        3: sum w |u|^2
//   4: sum w k2 |u|^2              5: sum w |u|^2 over the band
template <typename T>
__global__ void __launch_bounds__(NT) k_adj_sums(AdjArgs<T> a) {
  __shared__ double red[96];
  const Geom& g = a.g;
  const long long nm = (long long)g.Nx * g.Ny * g.Nzh;
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < nm; m += (long long)gridDim.x * NT) {
    int fx, fy, z;
    const Mode<T> d = mode_of(m, g, a.k, fx, fy, z);
    V2<T> u[3], v[3], pv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      u[c] = a.u[c * nm + m];
      v[c] = a.v[c * nm + m];
      pv[c] = v[c];
    }
    proj_mask(d, pv);
    const bool band = a.kmin2 <= d.k2 && d.k2 <= a.kmax2;
    const double pu = re_dot3<T>(pv, u), u2 = re_dot3<T>(u, u);
    s[0] += pu;
    if (band) s[1] += pu;
    s[2] += (double)d.k2 * re_dot3<T>(v, u);
    s[3] += d.w * u2;
    s[4] += d.w * (double)d.k2 * u2;
    if (band) s[5] += d.w * u2;
  }
  block_sum3_f64(s[0], s[1], s[2], red);
  if (threadIdx.x == 0) {
    a.partial[6 * blockIdx.x + 0] = s[0];
    a.partial[6 * blockIdx.x + 1] = s[1];
    a.partial[6 * blockIdx.x + 2] = s[2];
  }
  block_sum3_f64(s[3], s[4], s[5], red);
  if (threadIdx.x == 0) {
    a.partial[6 * blockIdx.x + 3] = s[3];
    a.partial[6 * blockIdx.x + 4] = s[4];
    a.partial[6 * blockIdx.x + 5] = s[5];
  }
}

// Scalars of the forcing transpose from the six sums (one thread):
//   scal[0] a_all  (pv coefficient, every mode)   scal[1] a_band (pv coefficient, band)
//   scal[2] c_w    (coefficient of w u)           scal[3] c_wk2  (of w k2 u)
//   scal[4] c_wb   (of w u over the band)
// and the parameter cotangents pct[0] nu, pct[1] A, pct[2] eps (added).
__global__ void k_adj_coef(AdjCoefArgs a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double* s = a.sums;
  const double n2 = a.ntot2;
  double sc[5] = {0, 0, 0, 0, 0};
  double dnu = -s[2], dA = 0.0, deps = 0.0;
  if (a.forcing == 1) {  // f = A u (forcing.py:94-95)
    sc[0] = a.A;
    dA = s[0];
  } else if (a.forcing == 2) {  // f = c mask u, c = eps / 2E_band (forcing.py:138-143)
    const double twoE = s[5] / n2;
    if (twoE > a.tiny) {
      const double c = a.eps / twoE;
      sc[1] = c;
      sc[4] = s[1] * (-c / twoE) * 2.0 / n2;
      deps = s[1] / twoE;
    }
  } else if (a.forcing == 3) {  // f = A(u) u, A = (2 nu Omega - (E - E_t)/tau) / 2E
    const double E = s[3] / (2.0 * n2), Om = s[4] / (2.0 * n2);
    if (E > 0.0) {
      const double itau = (a.tau > 0.0 && isfinite(a.tau)) ? 1.0 / a.tau : 0.0;
      const double relax = (a.tau > 0.0 && isfinite(a.tau)) ? (E - a.E_target) / a.tau : 0.0;
      const double A = (2.0 * a.nu * Om - relax) / (2.0 * E);
      const double beta = s[0];
      sc[0] = A;
      sc[2] = beta / n2 * (-itau / (2.0 * E) - A / E);
      sc[3] = beta / n2 * (a.nu / E);
      dnu += beta * Om / E;
    }
  }
  for (int i = 0; i < 5; ++i) a.scal[i] = sc[i];
  a.pct[0] += dnu;
  a.pct[1] += dA;
  a.pct[2] += deps;
}

// Per mode: the transform inputs X9 = [u, 1j k x u, pv / w] and the pointwise
// part of the cotangent ub = -nu k2 v + forcing terms.
template <typename T>
__global__ void __launch_bounds__(NT) k_adj_prep(AdjArgs<T> a) {
  const Geom& g = a.g;
  const long long nm = (long long)g.Nx * g.Ny * g.Nzh;
  const double* sc = a.scal;
  const T a_all = (T)sc[0], a_band = (T)sc[1], c_w = (T)sc[2], c_wk2 = (T)sc[3], c_wb = (T)sc[4];
  for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < nm; m += (long long)gridDim.x * NT) {
    int fx, fy, z;
    const Mode<T> d = mode_of(m, g, a.k, fx, fy, z);
    V2<T> u[3], v[3], pv[3], cu[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      u[c] = a.u[c * nm + m];
      v[c] = a.v[c * nm + m];
      pv[c] = v[c];
    }
    proj_mask(d, pv);
    curl_of(d, u, cu);
    const bool band = a.kmin2 <= d.k2 && d.k2 <= a.kmax2;
    const T iw = T(1) / (T)d.w;  // 1 or 1/2: exact
    const T ap = a_all + (band ? a_band : T(0));
    const T cu_ = (T)d.w * (c_w + d.k2 * c_wk2 + (band ? c_wb : T(0)));
    const T nk2 = a.nu * d.k2;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      a.x9[c * nm + m] = u[c];
      a.x9[(3 + c) * nm + m] = cu[c];
      a.x9[(6 + c) * nm + m] = cscale(pv[c], iw);
      V2<T> ub;
      ub.x = -nk2 * v[c].x + ap * pv[c].x + cu_ * u[c].x;
      ub.y = -nk2 * v[c].y + ap * pv[c].y + cu_ * u[c].y;
      a.ub[c * nm + m] = ub;
    }
  }
}

// Physical points: (u, om, g) in p[0..8] -> om x g into p[3..5], g x u into p[6..8].
template <typename T>
__global__ void __launch_bounds__(NT) k_adj_cross(T* __restrict__ p, long long n) {
  for (long long i = blockIdx.x * (long long)NT + threadIdx.x; i < n; i += (long long)gridDim.x * NT) {
    const T u0 = p[i], u1 = p[n + i], u2 = p[2 * n + i];
    const T o0 = p[3 * n + i], o1 = p[4 * n + i], o2 = p[5 * n + i];
    const T g0 = p[6 * n + i], g1 = p[7 * n + i], g2 = p[8 * n + i];
    p[3 * n + i] = o1 * g2 - o2 * g1;
    p[4 * n + i] = o2 * g0 - o0 * g2;
    p[5 * n + i] = o0 * g1 - o1 * g0;
    p[6 * n + i] = g1 * u2 - g2 * u1;
    p[7 * n + i] = g2 * u0 - g0 * u2;
    p[8 * n + i] = g0 * u1 - g1 * u0;
  }
}

// ub += w (s6[0..2] + 1j k x s6[3..5])
template <typename T>
__global__ void __launch_bounds__(NT) k_adj_combine(AdjArgs<T> a) {
  const Geom& g = a.g;
  const long long nm = (long long)g.Nx * g.Ny * g.Nzh;
  for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < nm; m += (long long)gridDim.x * NT) {
    int fx, fy, z;
    const Mode<T> d = mode_of(m, g, a.k, fx, fy, z);
    V2<T> A[3], B[3], cb[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      A[c] = a.s6[c * nm + m];
      B[c] = a.s6[(3 + c) * nm + m];
    }
    curl_of(d, B, cb);
    const T w = (T)d.w;
#pragma unroll
    for (int c = 0; c < 3; ++c) a.ub[c * nm + m] = cadd(a.ub[c * nm + m], cscale(cadd(A[c], cb[c]), w));
  }
}

// out = alpha x + beta y over n complex values (y may be NULL when beta = 0)
template <typename T>
__global__ void __launch_bounds__(NT) k_axpby(const V2<T>* __restrict__ x, T alpha, const V2<T>* __restrict__ y, T beta,
                                             V2<T>* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)NT + threadIdx.x; i < n; i += (long long)gridDim.x * NT) {
    V2<T> r = cscale(x[i], alpha);
    if (y) r = cadd(r, cscale(y[i], beta));
    out[i] = r;
  }
}

template <typename T> cudaError_t launch_adj_sums(const AdjArgs<T>& a, int nblocks, cudaStream_t st) {
  k_adj_sums<T><<<nblocks, NT, 0, st>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_adj_coef(const AdjCoefArgs& a, cudaStream_t st) {
  k_adj_coef<<<1, 32, 0, st>>>(a);
  return cudaGetLastError();
}
template <typename T> cudaError_t launch_adj_prep(const AdjArgs<T>& a, cudaStream_t st) {
  k_adj_prep<T><<<grid_of((long long)a.g.Nx * a.g.Ny * a.g.Nzh), NT, 0, st>>>(a);
  return cudaGetLastError();
}
template <typename T> cudaError_t launch_adj_cross(T* p, long long n, cudaStream_t st) {
  k_adj_cross<T><<<grid_of(n), NT, 0, st>>>(p, n);
  return cudaGetLastError();
}
template <typename T> cudaError_t launch_adj_combine(const AdjArgs<T>& a, cudaStream_t st) {
  k_adj_combine<T><<<grid_of((long long)a.g.Nx * a.g.Ny * a.g.Nzh), NT, 0, st>>>(a);
  return cudaGetLastError();
}
template <typename T>
cudaError_t launch_axpby(const V2<T>* x, T alpha, const V2<T>* y, T beta, V2<T>* out, long long n, cudaStream_t st) {
  k_axpby<T><<<grid_of(n), NT, 0, st>>>(x, alpha, y, beta, out, n);
  return cudaGetLastError();
}

template cudaError_t launch_adj_sums<float>(const AdjArgs<float>&, int, cudaStream_t);
template cudaError_t launch_adj_sums<double>(const AdjArgs<double>&, int, cudaStream_t);
template cudaError_t launch_adj_prep<float>(const AdjArgs<float>&, cudaStream_t);
template cudaError_t launch_adj_prep<double>(const AdjArgs<double>&, cudaStream_t);
template cudaError_t launch_adj_cross<float>(float*, long long, cudaStream_t);
template cudaError_t launch_adj_cross<double>(double*, long long, cudaStream_t);
template cudaError_t launch_adj_combine<float>(const AdjArgs<float>&, cudaStream_t);
template cudaError_t launch_adj_combine<double>(const AdjArgs<double>&, cudaStream_t);
template cudaError_t launch_axpby<float>(const float2*, float, const float2*, float, float2*, long long, cudaStream_t);
template cudaError_t launch_axpby<double>(const double2*, double, const double2*, double, double2*, long long,
                                          cudaStream_t);

}  // namespace hit

namespace hit {
// ---------------------------------------------------------------------------
// LES with the learned closure (no reference counterpart)
// ---------------------------------------------------------------------------

// g[3i + j] = 1j k_j u_i (spectral velocity gradients, 9 components)
template <typename T>
__global__ void __launch_bounds__(NT) k_grad9(const V2<T>* __restrict__ u, V2<T>* __restrict__ g, Geom gm, KTab<T> kt) {
  const long long nm = (long long)gm.Nx * gm.Ny * gm.Nzh;
  for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < nm; m += (long long)gridDim.x * NT) {
    const int z = (int)(m % gm.Nzh);
    const long long r = m / gm.Nzh;
    const int fy = (int)(r % gm.Ny), fx = (int)(r / gm.Ny);
    const T k[3] = {kt.kx[fx], kt.ky[fy], kt.kz[z]};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const V2<T> ui = u[i * nm + m];
#pragma unroll
      for (int j = 0; j < 3; ++j) g[(3 * i + j) * nm + m] = cmul_i(cscale(ui, k[j]));
    }
  }
}

// du += project(dealias(-1j k_j tau_ij)), tau in the order xx, yy, zz, xy, xz, yz
template <typename T, bool ADD>
__global__ void __launch_bounds__(NT) k_sgs_force(const V2<T>* __restrict__ t, V2<T>* __restrict__ du, Geom gm,
                                                  KTab<T> kt) {
  const long long nm = (long long)gm.Nx * gm.Ny * gm.Nzh;
  for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < nm; m += (long long)gridDim.x * NT) {
    int fx, fy, z;
    const Mode<T> d = mode_of(m, gm, kt, fx, fy, z);
    const V2<T> xx = t[m], yy = t[nm + m], zz = t[2 * nm + m], xy = t[3 * nm + m], xz = t[4 * nm + m],
                yz = t[5 * nm + m];
    V2<T> f[3];
    // k_j tau_ij, then times -1j
    V2<T> s0, s1, s2;
    s0.x = d.kx * xx.x + d.ky * xy.x + d.kz * xz.x;
    s0.y = d.kx * xx.y + d.ky * xy.y + d.kz * xz.y;
    s1.x = d.kx * xy.x + d.ky * yy.x + d.kz * yz.x;
    s1.y = d.kx * xy.y + d.ky * yy.y + d.kz * yz.y;
    s2.x = d.kx * xz.x + d.ky * yz.x + d.kz * zz.x;
    s2.y = d.kx * xz.y + d.ky * yz.y + d.kz * zz.y;
    f[0] = cmul_mi(s0);
    f[1] = cmul_mi(s1);
    f[2] = cmul_mi(s2);
    proj_mask(d, f);
#pragma unroll
    for (int c = 0; c < 3; ++c) du[c * nm + m] = ADD ? cadd(du[c * nm + m], f[c]) : f[c];
  }
}

// Transpose of k_sgs_force (the write form f = P(-1j K tau_hat), P the
// dealias mask and projection, (K tau_hat)_i = k_j tau_hat_ij with the
// symmetric tau in the order xx, yy, zz, xy, xz, yz).  Cotangents are
// dL/dRe + i dL/dIm of each stored entry, so a per-mode complex-linear map
// transposes to its conjugate transpose: g = P fbar (P is real symmetric per
// mode), h = 1j g, tau_hat_bar = K^T h.  Written times scale / w (w the
// Hermitian weight of the mode's plane): with scale = Nx Ny Nz the c2r of the
// result is the cotangent of the physical stress, because the transpose of
// rfftn is N^3 irfftn(. / w).
template <typename T>
__global__ void __launch_bounds__(NT) k_sgs_force_vjp(const V2<T>* __restrict__ fb, V2<T>* __restrict__ tb, Geom gm,
                                                      KTab<T> kt, T scale) {
  const long long nm = (long long)gm.Nx * gm.Ny * gm.Nzh;
  for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < nm; m += (long long)gridDim.x * NT) {
    int fx, fy, z;
    const Mode<T> d = mode_of(m, gm, kt, fx, fy, z);
    V2<T> h[3] = {fb[m], fb[nm + m], fb[2 * nm + m]};
    proj_mask(d, h);
    const T c = scale / (T)d.w;
#pragma unroll
    for (int i = 0; i < 3; ++i) h[i] = cscale(cmul_i(h[i]), c);
    tb[m] = cscale(h[0], d.kx);
    tb[nm + m] = cscale(h[1], d.ky);
    tb[2 * nm + m] = cscale(h[2], d.kz);
    tb[3 * nm + m] = cadd(cscale(h[0], d.ky), cscale(h[1], d.kx));
    tb[4 * nm + m] = cadd(cscale(h[0], d.kz), cscale(h[2], d.kx));
    tb[5 * nm + m] = cadd(cscale(h[1], d.kz), cscale(h[2], d.ky));
  }
}

// Transpose of the velocity gradients g_(3i+j) = irfftn(1j k_j u_hat_i): with
// G the rfftn of the 9 physical gradient cotangents, u_bar_i += sum_j
// (-1j k_j) (w / N^3) G_ij (the transpose of irfftn is w rfftn(.) / N^3).
template <typename T>
__global__ void __launch_bounds__(NT) k_grad9_vjp(const V2<T>* __restrict__ G, V2<T>* __restrict__ ub, Geom gm,
                                                  KTab<T> kt, T inv_n3) {
  const long long nm = (long long)gm.Nx * gm.Ny * gm.Nzh;
  for (long long m = blockIdx.x * (long long)NT + threadIdx.x; m < nm; m += (long long)gridDim.x * NT) {
    const int z = (int)(m % gm.Nzh);
    const long long r = m / gm.Nzh;
    const int fy = (int)(r % gm.Ny), fx = (int)(r / gm.Ny);
    const T k[3] = {kt.kx[fx], kt.ky[fy], kt.kz[z]};
    const T c = (T)herm_weight(gm, z) * inv_n3;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      V2<T> s = czero<T>();
#pragma unroll
      for (int j = 0; j < 3; ++j) s = cadd(s, cscale(G[(3 * i + j) * nm + m], k[j]));
      ub[i * nm + m] = cadd(ub[i * nm + m], cscale(cmul_mi(s), c));
    }
  }
}

template <typename T>
cudaError_t launch_sgs_force_vjp(const V2<T>* fb, V2<T>* tb, const Geom& gm, KTab<T> kt, T scale, cudaStream_t st) {
  k_sgs_force_vjp<T><<<grid_of((long long)gm.Nx * gm.Ny * gm.Nzh), NT, 0, st>>>(fb, tb, gm, kt, scale);
  return cudaGetLastError();
}
template <typename T>
cudaError_t launch_grad9_vjp(const V2<T>* G, V2<T>* ub, const Geom& gm, KTab<T> kt, T inv_n3, cudaStream_t st) {
  k_grad9_vjp<T><<<grid_of((long long)gm.Nx * gm.Ny * gm.Nzh), NT, 0, st>>>(G, ub, gm, kt, inv_n3);
  return cudaGetLastError();
}
template cudaError_t launch_sgs_force_vjp<float>(const float2*, float2*, const Geom&, KTab<float>, float, cudaStream_t);
template cudaError_t launch_sgs_force_vjp<double>(const double2*, double2*, const Geom&, KTab<double>, double,
                                                  cudaStream_t);
template cudaError_t launch_grad9_vjp<float>(const float2*, float2*, const Geom&, KTab<float>, float, cudaStream_t);
template cudaError_t launch_grad9_vjp<double>(const double2*, double2*, const Geom&, KTab<double>, double,
                                              cudaStream_t);

template <typename T> cudaError_t launch_grad9(const V2<T>* u, V2<T>* g, const Geom& gm, KTab<T> kt, cudaStream_t st) {
  k_grad9<T><<<grid_of((long long)gm.Nx * gm.Ny * gm.Nzh), NT, 0, st>>>(u, g, gm, kt);
  return cudaGetLastError();
}
template <typename T>
cudaError_t launch_sgs_force(const V2<T>* t, V2<T>* du, const Geom& gm, KTab<T> kt, cudaStream_t st, bool add) {
  if (add) k_sgs_force<T, true><<<grid_of((long long)gm.Nx * gm.Ny * gm.Nzh), NT, 0, st>>>(t, du, gm, kt);
  else k_sgs_force<T, false><<<grid_of((long long)gm.Nx * gm.Ny * gm.Nzh), NT, 0, st>>>(t, du, gm, kt);
  return cudaGetLastError();
}
template cudaError_t launch_grad9<float>(const float2*, float2*, const Geom&, KTab<float>, cudaStream_t);
template cudaError_t launch_grad9<double>(const double2*, double2*, const Geom&, KTab<double>, cudaStream_t);
template cudaError_t launch_sgs_force<float>(const float2*, float2*, const Geom&, KTab<float>, cudaStream_t, bool);
template cudaError_t launch_sgs_force<double>(const double2*, double2*, const Geom&, KTab<double>, cudaStream_t, bool);
}  // namespace hit
