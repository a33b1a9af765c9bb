// z-axis (contiguous, rfft-halved) kernels.
//
// The real transforms along z use one complex FFT of length H = Nz/2 per row:
//   c2r: Z[k] = (X[k] + conj X[H-k]) + i e^{+2 pi i k/Nz} (X[k] - conj X[H-k]),
//        z = IFFT_H(Z), x[2m] = Re z[m], x[2m+1] = Im z[m]   (times 1/N);
//        the imaginary parts of X[0] and X[H] are dropped first, which is the
//        numpy/pocketfft irfft convention the reference inherits
//        (src/hit3d/grid.py:181-183: complex inverses over x, y, then c2r on z).
//   r2c: z[m] = x[2m] + i x[2m+1], Z = FFT_H(z),
//        X[k] = (Z[k] + conj Z[H-k])/2 - i e^{-2 pi i k/Nz} (Z[k] - conj Z[H-k])/2.
//
// k_zcross fuses the middle of the RHS (src/hit3d/navierstokes.py:78-89): c2r of
// u and w (6 rows), the pointwise u x w in physical space, r2c of the 3
// products, all in shared memory, writing the products over the first three
// input components of the same rows.
#include <type_traits>

#include "fft_core.cuh"
#include "kernels.h"

namespace hit {

template <int H> constexpr int z_rows_per_block() { return (1024 / H) > 32 ? 32 : (1024 / H < 1 ? 1 : 1024 / H); }

// conj-paired pre-processing of one c2r row element k in [0, H).
template <typename T>
__device__ __forceinline__ V2<T> c2r_pre(const V2<T>* row, int k, int H, int Mz, const V2<T>* tw, int twstep) {
  V2<T> X = k < Mz ? row[k] : czero<T>();
  const int kk = H - k;  // in [1, H]
  V2<T> Y = kk < Mz ? row[kk] : czero<T>();
  if (k == 0) {
    X.y = T(0);
    Y.y = T(0);  // kk == H: Nyquist
  }
  Y.y = -Y.y;  // conj X[H-k]
  const V2<T> s = cadd(X, Y), d = csub(X, Y);
  V2<T> w = __ldg(&tw[k * twstep]);
  w.y = -w.y;  // e^{+2 pi i k / Nz}
  return cadd(s, cmul_i(cmul(w, d)));
}

// r2c post-processing: output bin k in [0, H] from Z (length H, row stride 1).
template <typename T>
__device__ __forceinline__ V2<T> r2c_post(const V2<T>* Z, int k, int H, const V2<T>* tw, int twstep) {
  const V2<T> a = Z[k == H ? 0 : k];
  V2<T> b = Z[k == 0 ? 0 : H - k];
  b.y = -b.y;
  const V2<T> E = cscale(cadd(a, b), T(0.5));
  const V2<T> O = cmul_mi(cscale(csub(a, b), T(0.5)));
  const V2<T> w = __ldg(&tw[k * twstep]);  // e^{-2 pi i k / Nz}
  return cadd(E, cmul(w, O));
}

template <typename T, int H, int RB>
__global__ void __launch_bounds__(NT) k_zcross(ZCrossArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int LD = H + 1;
  constexpr int twstep = TWN / (2 * H);
  V2<T>* Z = reinterpret_cast<V2<T>*>(smem_raw);  // [6*RB][LD]
  const long long row0 = (long long)blockIdx.x * RB;

  for (int e = threadIdx.x; e < 6 * RB * H; e += NT) {
    const int q = e / (RB * H), rem = e % (RB * H), lr = rem / H, k = rem % H;
    const long long row = row0 + lr;
    V2<T> v = czero<T>();
    if (row < a.nrows) v = c2r_pre<T>(a.buf + q * a.c_stride + row * a.Mzp, k, H, a.Mz, a.tw, twstep);
    Z[(q * RB + lr) * LD + k] = v;
  }
  __syncthreads();
  smem_fft<T, H, 6 * RB, NT, 1, LD, true>(Z, a.tw);

  // u x w in physical space (navierstokes.py:82-86), on both halves of each pair
  for (int e = threadIdx.x; e < RB * H; e += NT) {
    const int lr = e / H, m = e % H;
    V2<T> u[3], w[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      u[c] = cscale(Z[(c * RB + lr) * LD + m], a.scale);
      w[c] = cscale(Z[((3 + c) * RB + lr) * LD + m], a.scale);
    }
    V2<T> n0, n1, n2;
    n0.x = u[1].x * w[2].x - u[2].x * w[1].x;
    n0.y = u[1].y * w[2].y - u[2].y * w[1].y;
    n1.x = u[2].x * w[0].x - u[0].x * w[2].x;
    n1.y = u[2].y * w[0].y - u[0].y * w[2].y;
    n2.x = u[0].x * w[1].x - u[1].x * w[0].x;
    n2.y = u[0].y * w[1].y - u[1].y * w[0].y;
    Z[(0 * RB + lr) * LD + m] = n0;
    Z[(1 * RB + lr) * LD + m] = n1;
    Z[(2 * RB + lr) * LD + m] = n2;
  }
  __syncthreads();
  smem_fft<T, H, 3 * RB, NT, 1, LD, false>(Z, a.tw);

  for (int e = threadIdx.x; e < 3 * RB * a.Mzp; e += NT) {
    const int q = e / (RB * a.Mzp), rem = e % (RB * a.Mzp), lr = rem / a.Mzp, k = rem % a.Mzp;
    const long long row = row0 + lr;
    if (row < a.nrows) {
      V2<T> v = czero<T>();
      if (k < a.Mz) v = r2c_post<T>(Z + (q * RB + lr) * LD, k, H, a.tw, twstep);
      a.buf[q * a.c_stride + row * a.Mzp + k] = v;
    }
  }
}

template <typename T, int H, int RB>
__global__ void __launch_bounds__(NT) k_zc2r(ZRealArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int LD = H + 1;
  constexpr int twstep = TWN / (2 * H);
  V2<T>* Z = reinterpret_cast<V2<T>*>(smem_raw);
  const long long row0 = (long long)blockIdx.x * RB;
  const long long c = blockIdx.y;
  for (int e = threadIdx.x; e < RB * H; e += NT) {
    const int lr = e / H, k = e % H;
    const long long row = row0 + lr;
    V2<T> v = czero<T>();
    if (row < a.nrows) v = c2r_pre<T>(a.cbuf + c * a.cc_stride + row * a.Mzp, k, H, a.Mz, a.tw, twstep);
    Z[lr * LD + k] = v;
  }
  __syncthreads();
  smem_fft<T, H, RB, NT, 1, LD, true>(Z, a.tw);
  for (int e = threadIdx.x; e < RB * H; e += NT) {
    const int lr = e / H, m = e % H;
    const long long row = row0 + lr;
    if (row < a.nrows) {
      V2<T>* out = reinterpret_cast<V2<T>*>(a.rbuf + c * a.rc_stride + row * (2 * H));
      out[m] = cscale(Z[lr * LD + m], a.scale);
    }
  }
}

template <typename T, int H, int RB>
__global__ void __launch_bounds__(NT) k_zr2c(ZRealArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int LD = H + 1;
  constexpr int twstep = TWN / (2 * H);
  V2<T>* Z = reinterpret_cast<V2<T>*>(smem_raw);
  const long long row0 = (long long)blockIdx.x * RB;
  const long long c = blockIdx.y;
  for (int e = threadIdx.x; e < RB * H; e += NT) {
    const int lr = e / H, m = e % H;
    const long long row = row0 + lr;
    V2<T> v = czero<T>();
    if (row < a.nrows) v = reinterpret_cast<const V2<T>*>(a.rbuf + c * a.rc_stride + row * (2 * H))[m];
    Z[lr * LD + m] = v;
  }
  __syncthreads();
  smem_fft<T, H, RB, NT, 1, LD, false>(Z, a.tw);
  for (int e = threadIdx.x; e < RB * a.Mzp; e += NT) {
    const int lr = e / a.Mzp, k = e % a.Mzp;
    const long long row = row0 + lr;
    if (row < a.nrows) {
      V2<T> v = czero<T>();
      if (k < a.Mz) v = r2c_post<T>(Z + lr * LD, k, H, a.tw, twstep);
      a.cbuf[c * a.cc_stride + row * a.Mzp + k] = v;
    }
  }
}

template <typename F> cudaError_t dispatch_half(int H, F&& f) {
  switch (H) {
    case 2: return f(std::integral_constant<int, 2>{});
    case 4: return f(std::integral_constant<int, 4>{});
    case 8: return f(std::integral_constant<int, 8>{});
    case 16: return f(std::integral_constant<int, 16>{});
    case 32: return f(std::integral_constant<int, 32>{});
    case 64: return f(std::integral_constant<int, 64>{});
    case 128: return f(std::integral_constant<int, 128>{});
    case 256: return f(std::integral_constant<int, 256>{});
    case 512: return f(std::integral_constant<int, 512>{});
    default: return cudaErrorInvalidValue;
  }
}

template <typename T> cudaError_t launch_zcross(int H, const ZCrossArgs<T>& a, cudaStream_t st) {
  return dispatch_half(H, [&](auto hh) {
    constexpr int HH = decltype(hh)::value;
    constexpr int RB = z_rows_per_block<HH>();
    const size_t smem = sizeof(V2<T>) * 6 * RB * (HH + 1);
    const int nb = (a.nrows + RB - 1) / RB;
    k_zcross<T, HH, RB><<<nb, NT, smem, st>>>(a);
    return cudaGetLastError();
  });
}

template <typename T> cudaError_t launch_zc2r(int H, const ZRealArgs<T>& a, int ncomp, cudaStream_t st) {
  return dispatch_half(H, [&](auto hh) {
    constexpr int HH = decltype(hh)::value;
    constexpr int RB = z_rows_per_block<HH>();
    const size_t smem = sizeof(V2<T>) * RB * (HH + 1);
    dim3 grid((a.nrows + RB - 1) / RB, ncomp);
    k_zc2r<T, HH, RB><<<grid, NT, smem, st>>>(a);
    return cudaGetLastError();
  });
}

template <typename T> cudaError_t launch_zr2c(int H, const ZRealArgs<T>& a, int ncomp, cudaStream_t st) {
  return dispatch_half(H, [&](auto hh) {
    constexpr int HH = decltype(hh)::value;
    constexpr int RB = z_rows_per_block<HH>();
    const size_t smem = sizeof(V2<T>) * RB * (HH + 1);
    dim3 grid((a.nrows + RB - 1) / RB, ncomp);
    k_zr2c<T, HH, RB><<<grid, NT, smem, st>>>(a);
    return cudaGetLastError();
  });
}

template <typename T> cudaError_t prepare_axis_kernels(int Nx);

template <typename T> cudaError_t prepare_fft_kernels(int Nx, int Ny, int Nz) {
  (void)Ny;
  cudaError_t e = prepare_axis_kernels<T>(Nx);
  if (e != cudaSuccess) return e;
  return dispatch_half(Nz / 2, [&](auto hh) {
    constexpr int HH = decltype(hh)::value;
    constexpr int RB = z_rows_per_block<HH>();
    const int smem = (int)(sizeof(V2<T>) * 6 * RB * (HH + 1));
    return cudaFuncSetAttribute(k_zcross<T, HH, RB>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  });
}

template cudaError_t launch_zcross<float>(int, const ZCrossArgs<float>&, cudaStream_t);
template cudaError_t launch_zcross<double>(int, const ZCrossArgs<double>&, cudaStream_t);
template cudaError_t launch_zc2r<float>(int, const ZRealArgs<float>&, int, cudaStream_t);
template cudaError_t launch_zc2r<double>(int, const ZRealArgs<double>&, int, cudaStream_t);
template cudaError_t launch_zr2c<float>(int, const ZRealArgs<float>&, int, cudaStream_t);
template cudaError_t launch_zr2c<double>(int, const ZRealArgs<double>&, int, cudaStream_t);
template cudaError_t prepare_fft_kernels<float>(int, int, int);
template cudaError_t prepare_fft_kernels<double>(int, int, int);

}  // namespace hit
