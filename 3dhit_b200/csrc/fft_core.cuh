// In-shared-memory batched complex FFT (Stockham, decimation in time) for
// power-of-two lengths 2..1024.  Radix plan: one radix-2 or radix-4 stage when
// log2(N) is not a multiple of 3, then radix-8 stages.  Each thread owns whole
// butterflies: it loads all of its butterfly inputs for a stage into
// registers, the block synchronises, then it twiddles, runs the radix-R DFT in
// registers and stores in place.  Twiddles come from a host table of
// exp(-2 pi i m / TWN) rounded from long double, so no device sin/cos is used.
//
// Element (pos, col) of the batch lives at buf[pos*SP + col*SC]; SP/SC let the
// same code transform strided column tiles (x, y passes) and contiguous rows
// (z pass).
#pragma once

#include "common.cuh"

namespace hit {

constexpr int TWN = 2048;  // twiddle table length (supports N <= 2048)

__host__ __device__ constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n >> 1); }
__host__ __device__ constexpr int fft_nstages(int N) { return (ilog2(N) + 2) / 3; }
__host__ __device__ constexpr int fft_radix(int N, int s) {
  return (ilog2(N) % 3 != 0 && s == 0) ? (ilog2(N) % 3 == 1 ? 2 : 4) : 8;
}
__host__ __device__ constexpr int fft_pprod(int N, int s) { return s == 0 ? 1 : fft_pprod(N, s - 1) * fft_radix(N, s - 1); }

template <bool INV, typename V> __device__ __forceinline__ void dft4(V& x0, V& x1, V& x2, V& x3) {
  V a = cadd(x0, x2), b = csub(x0, x2), c = cadd(x1, x3), d = csub(x1, x3);
  d = INV ? cmul_i(d) : cmul_mi(d);
  x0 = cadd(a, c);
  x2 = csub(a, c);
  x1 = cadd(b, d);
  x3 = csub(b, d);
}

template <int R, bool INV, typename V> struct DFT;
template <bool INV, typename V> struct DFT<2, INV, V> {
  static __device__ __forceinline__ void run(V* v) {
    V a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};
template <bool INV, typename V> struct DFT<4, INV, V> {
  static __device__ __forceinline__ void run(V* v) { dft4<INV>(v[0], v[1], v[2], v[3]); }
};
template <bool INV, typename V> struct DFT<8, INV, V> {
  static __device__ __forceinline__ void run(V* v) {
    using T = decltype(v[0].x);
    const T h = T(0.70710678118654752440084436210484903928);  // sqrt(2)/2
    V e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    V o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<INV>(e0, e1, e2, e3);
    dft4<INV>(o0, o1, o2, o3);
    // o_k *= W8^{k} (W8 = exp(-+ i pi/4))
    V t1, t2, t3;
    if (!INV) {
      t1.x = (o1.x + o1.y) * h; t1.y = (o1.y - o1.x) * h;   // (1-i)/sqrt2
      t2 = cmul_mi(o2);                                      // -i
      t3.x = (o3.y - o3.x) * h; t3.y = -(o3.x + o3.y) * h;  // (-1-i)/sqrt2
    } else {
      t1.x = (o1.x - o1.y) * h; t1.y = (o1.x + o1.y) * h;   // (1+i)/sqrt2
      t2 = cmul_i(o2);                                       // +i
      t3.x = -(o3.x + o3.y) * h; t3.y = (o3.x - o3.y) * h;  // (-1+i)/sqrt2
    }
    v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
    v[1] = cadd(e1, t1); v[5] = csub(e1, t1);
    v[2] = cadd(e2, t2); v[6] = csub(e2, t2);
    v[3] = cadd(e3, t3); v[7] = csub(e3, t3);
  }
};

// One Stockham stage: radix R, P = product of the previous radices.
template <typename T, int N, int NCOLS, int NT, int SP, int SC, bool INV, int R, int P>
__device__ __forceinline__ void fft_stage(V2<T>* __restrict__ buf, const V2<T>* __restrict__ tw) {
  constexpr int NB = N / R;
  constexpr int TOTAL = NB * NCOLS;
  constexpr int CNT = (TOTAL + NT - 1) / NT;
  V2<T> v[CNT][R];
#pragma unroll
  for (int c = 0; c < CNT; ++c) {
    const int t = threadIdx.x + c * NT;
    if (TOTAL % NT == 0 || t < TOTAL) {
      const int col = t % NCOLS, b = t / NCOLS;
#pragma unroll
      for (int r = 0; r < R; ++r) v[c][r] = buf[(b + r * NB) * SP + col * SC];
    }
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < CNT; ++c) {
    const int t = threadIdx.x + c * NT;
    if (TOTAL % NT == 0 || t < TOTAL) {
      const int col = t % NCOLS, b = t / NCOLS;
      const int k = b & (P - 1);
      if (P > 1) {
        constexpr int STEP = (TWN / N) * (N / (P * R));
#pragma unroll
        for (int r = 1; r < R; ++r) {
          V2<T> w = __ldg(&tw[r * k * STEP]);
          if (INV) w.y = -w.y;
          v[c][r] = cmul(v[c][r], w);
        }
      }
      DFT<R, INV, V2<T>>::run(v[c]);
      const int j = (b - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) buf[(j + r * P) * SP + col * SC] = v[c][r];
    }
  }
  __syncthreads();
}

template <typename T, int N, int NCOLS, int NT, int SP, int SC, bool INV, int S>
__device__ __forceinline__ void fft_stages(V2<T>* buf, const V2<T>* tw) {
  if constexpr (S < fft_nstages(N)) {
    fft_stage<T, N, NCOLS, NT, SP, SC, INV, fft_radix(N, S), fft_pprod(N, S)>(buf, tw);
    fft_stages<T, N, NCOLS, NT, SP, SC, INV, S + 1>(buf, tw);
  }
}

// Unnormalised in-place FFT of NCOLS sequences of length N held in shared
// memory.  Caller: __syncthreads() after filling buf; on return buf holds the
// transform and the block is synchronised.  INV selects exp(+2 pi i nk/N).
template <typename T, int N, int NCOLS, int NT, int SP, int SC, bool INV>
__device__ __forceinline__ void smem_fft(V2<T>* buf, const V2<T>* tw) {
  static_assert((N & (N - 1)) == 0 && N >= 2 && N <= TWN, "power-of-two length");
  fft_stages<T, N, NCOLS, NT, SP, SC, INV, 0>(buf, tw);
}

}  // namespace hit
