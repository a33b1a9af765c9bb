// Shared device helpers for the HIT3D sm_100a kernels: complex arithmetic on
// float2/double2, the plan geometry handed to every kernel, and the mapping
// between compact (pruned) spectral indices and full FFT positions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace hit {

template <typename T> struct VecOf;
template <> struct VecOf<float> { using type = float2; };
template <> struct VecOf<double> { using type = double2; };
template <typename T> using V2 = typename VecOf<T>::type;

template <typename T>
__host__ __device__ __forceinline__ V2<T> cx(T re, T im) {
  V2<T> r;
  r.x = re;
  r.y = im;
  return r;
}
template <typename T> __device__ __forceinline__ V2<T> czero() { return cx<T>(T(0), T(0)); }
template <typename V> __device__ __forceinline__ V cadd(V a, V b) { a.x += b.x; a.y += b.y; return a; }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename V> __device__ __forceinline__ V cconj(V a) { a.y = -a.y; return a; }
template <typename V> __device__ __forceinline__ V cmul(V a, V b) {
  V r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename V, typename T> __device__ __forceinline__ V cscale(V a, T s) { a.x *= s; a.y *= s; return a; }
// float2: one paired-FP32 instruction (FADD2 / FFMA2 / FMUL2) per complex
// add, subtract or scale; each component rounds exactly as the scalar
// operation does (a - b is formed as b * -1 + a, whose product is exact).
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
// multiply by +i / -i
template <typename V> __device__ __forceinline__ V cmul_i(V a) { V r; r.x = -a.y; r.y = a.x; return r; }
template <typename V> __device__ __forceinline__ V cmul_mi(V a) { V r; r.x = a.y; r.y = -a.x; return r; }

// Geometry of one call.  The spectral arrays a kernel touches are "compact":
// along x and y only M kept wavenumber rows are stored (the first h are the
// non-negative frequencies, the rest the negative ones), along z the first Mz
// of the Nz/2+1 rfft modes, with rows padded to Mzp.  With M = N, h = N/2 and
// Mz = Nz/2+1 the compact layout is the full reference layout (general path);
// with M = 2(N/3)+1, h = N/3+1 and Mz = Nz/3+1 it holds exactly the 2/3
// dealiasing box (dealiased path), so zero modes are never moved.
struct Geom {
  int Nx, Ny, Nz, H, Nzh;  // H = Nz/2, Nzh = Nz/2+1
  int Mx, hx, My, hy, Mz, Mzp;
  int cx, cy, cz;          // dealias cuts N_i/3
  int pruned;              // 1 when the compact set is the dealias box
};

// compact row index -> full FFT position (0..N-1)
__device__ __forceinline__ int full_pos(int i, int h, int M, int N) { return i < h ? i : i + N - M; }
// full FFT position -> compact row index, or -1 when the position is not stored
__device__ __forceinline__ int compact_row(int pos, int h, int M, int N) {
  if (pos < h) return pos;
  int off = N - M;
  return pos >= h + off ? pos - off : -1;
}
// fftfreq integer of a full position (N/2 maps to -N/2, as numpy.fft.fftfreq)
__device__ __forceinline__ int freq_of(int pos, int N) { return pos < N / 2 ? pos : pos - N; }

// 2/3-rule box (src/hit3d/grid.py:115-120): |nx|<=Nx/3, |ny|<=Ny/3, nz<=Nz/3, not k=0.
__device__ __forceinline__ bool in_dealias(const Geom& g, int fx, int fy, int kz) {
  int nx = freq_of(fx, g.Nx), ny = freq_of(fy, g.Ny);
  bool m = (abs(nx) <= g.cx) && (abs(ny) <= g.cy) && (kz <= g.cz);
  return m && !(fx == 0 && fy == 0 && kz == 0);
}

// Hermitian weight of an rfft plane (src/hit3d/grid.py:122-125).
__device__ __forceinline__ int herm_weight(const Geom& g, int kz) {
  return (kz == 0 || ((g.Nz & 1) == 0 && kz == g.H)) ? 1 : 2;
}

// |k|^2 exactly as the reference forms it in the run dtype: kx**2 + ky**2 + kz**2,
// each square and sum rounded separately (no FMA contraction).
__device__ __forceinline__ float k2_of(float kx, float ky, float kz) {
  return __fadd_rn(__fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky)), __fmul_rn(kz, kz));
}
__device__ __forceinline__ double k2_of(double kx, double ky, double kz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky)), __dmul_rn(kz, kz));
}
// 1/|k|^2 with 0 at k=0, correctly rounded (grid.py:110-111): the IEEE
// round-to-nearest reciprocal equals the correctly rounded quotient 1/k2.
__device__ __forceinline__ float inv_k2_of(float k2) { return k2 == 0.f ? 0.f : __frcp_rn(k2); }
__device__ __forceinline__ double inv_k2_of(double k2) { return k2 == 0.0 ? 0.0 : __drcp_rn(k2); }

// Integrating factor e^{-nu k^2 h} of the viscous operator -nu k^2
// (navierstokes.py:100-103) over a step h, in the run precision.
__device__ __forceinline__ float visc_factor(float nuh, float k2) { return expf(-nuh * k2); }
__device__ __forceinline__ double visc_factor(double nuh, double k2) { return exp(-nuh * k2); }

// Wavenumber tables (device): kx[Nx], ky[Ny], kz[Nzh], each value computed on the
// host as (T)(2*pi/L * n) in double, matching grid.py:101-107.
template <typename T> struct KTab {
  const T* kx;
  const T* ky;
  const T* kz;
};

// Programmatic dependent launch: a kernel launched with launch_pdl may start
// while the previous kernel in the stream is still finishing.  It sets up what
// depends on no earlier kernel (twiddle tables, shared-memory zero fill), then
// pdl_wait() returns once the previous grid has completed and its writes are
// visible; pdl_trigger() then lets the next kernel start launching.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

// Block-wide float64 sums of three values at once (all threads must call;
// blockDim.x a multiple of 32, scratch >= 96 doubles); valid in thread 0.
__device__ __forceinline__ void block_sum3_f64(double& a, double& b, double& c, double* scratch) {
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
    c += __shfl_xor_sync(0xffffffffu, c, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) {
    scratch[warp] = a;
    scratch[32 + warp] = b;
    scratch[64 + warp] = c;
  }
  __syncthreads();
  if (warp == 0) {
    a = lane < nw ? scratch[lane] : 0.0;
    b = lane < nw ? scratch[32 + lane] : 0.0;
    c = lane < nw ? scratch[64 + lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      b += __shfl_xor_sync(0xffffffffu, b, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
  }
}

// Block-wide float64 sum (all threads must call; blockDim.x a multiple of 32).
__device__ __forceinline__ double block_sum_f64(double v, double* scratch /*>= 32*/) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  int nw = blockDim.x >> 5;
  double r = 0.0;
  if (warp == 0) {
    r = lane < nw ? scratch[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  return r;  // valid in thread 0
}

}  // namespace hit
