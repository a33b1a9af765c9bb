// Batched complex FFT (Stockham, decimation in time) for power-of-two lengths
// 2..1024, with fused input and output.
//
// Radix plan: one radix-2 or radix-4 stage when log2(N) is not a multiple of
// 3, then radix-8 stages.  Each thread owns whole butterflies: it reads the R
// inputs of a butterfly, twiddles them, runs the radix-R DFT in registers and
// writes the R outputs.  Stage 0 reads through a loader functor ld(pos, col)
// (global memory, with zero padding, or a fused prologue); the last stage hands
// its outputs to a storer functor st(pos, col, v) (global memory, or a fused
// epilogue); the stages in between ping-pong between two shared-memory buffers
// A and B, with one barrier per stage boundary.  Twiddles come from a host
// table of exp(-2 pi i m / TWN) rounded from long double: no device sin/cos.
//
// Element (pos, col) of a shared buffer lives at buf[pos*SP + col*SC]; SP/SC let
// the same code transform strided column tiles (x, y passes) and contiguous
// rows (z pass).
#pragma once

#include <type_traits>

#include "common.cuh"

namespace hit {

constexpr int TWN = 2048;  // twiddle table length (supports N <= 2048)

__host__ __device__ constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n >> 1); }
// Radix-8 plan of the column transforms: radix-8 stages, with one radix-4
// first stage when log2(N) = 2 mod 3; when log2(N) = 1 mod 3 (N = 128, 1024)
// one radix-16 second stage (8 x 16 x 8 for 1024: the first and the last stage
// are radix 8, which the register-mode x-forward epilogue needs); N = 16 is
// 2 x 8.
__host__ __device__ constexpr bool fft_has16(int N) { return ilog2(N) % 3 == 1 && N >= 128; }
__host__ __device__ constexpr int fft_nstages(int N) { return fft_has16(N) ? (ilog2(N) - 1) / 3 : (ilog2(N) + 2) / 3; }
__host__ __device__ constexpr int fft_radix(int N, int s) {
  return fft_has16(N) ? (s == 1 ? 16 : 8) : ((ilog2(N) % 3 != 0 && s == 0) ? (ilog2(N) % 3 == 1 ? 2 : 4) : 8);
}
__host__ __device__ constexpr int fft_pprod(int N, int s) {
  return s == 0 ? 1 : fft_pprod(N, s - 1) * fft_radix(N, s - 1);
}
// Radix-16 plan (used by the in-place row FFTs): one radix-2/4/8 stage when
// log2(N) is not a multiple of 4, then radix-16 stages.
__host__ __device__ constexpr int fft16_nstages(int N) { return (ilog2(N) + 3) / 4; }
__host__ __device__ constexpr int fft16_radix(int N, int s) {
  return (ilog2(N) % 4 != 0 && s == 0) ? (1 << (ilog2(N) % 4)) : 16;
}
__host__ __device__ constexpr int fft16_pprod(int N, int s) {
  return s == 0 ? 1 : fft16_pprod(N, s - 1) * fft16_radix(N, s - 1);
}
template <bool PLAN16> __host__ __device__ constexpr int plan_nstages(int N) {
  return PLAN16 ? fft16_nstages(N) : fft_nstages(N);
}
template <bool PLAN16> __host__ __device__ constexpr int plan_radix(int N, int s) {
  return PLAN16 ? fft16_radix(N, s) : fft_radix(N, s);
}
template <bool PLAN16> __host__ __device__ constexpr int plan_pprod(int N, int s) {
  return PLAN16 ? fft16_pprod(N, s) : fft_pprod(N, s);
}
// Per-stage twiddle tables in shared memory: stage s >= 1 (radix R, P = product
// of the earlier radices) holds exp(-+2 pi i r k / (P R)) at slot
// off(s) + (r-1)*P + k, r in [1, R), k in [0, P): the lanes of a warp, which
// differ in k, read consecutive slots.
template <bool PLAN16> __host__ __device__ constexpr int tw_offset(int N, int s) {
  return s <= 1 ? 0 : tw_offset<PLAN16>(N, s - 1) + (plan_radix<PLAN16>(N, s - 1) - 1) * plan_pprod<PLAN16>(N, s - 1);
}
template <bool PLAN16> __host__ __device__ constexpr int tw_size(int N) {
  return plan_nstages<PLAN16>(N) < 2 ? 1 : tw_offset<PLAN16>(N, plan_nstages<PLAN16>(N));
}
// Fill the tables from the global exp(-2 pi i m / TWN) table (all threads call;
// the caller synchronises before first use).  Stage by stage, with the
// stage's radix, stride and offset as compile-time constants.
template <typename T, int N, bool PLAN16, int NTH, int S = 1>
__device__ __forceinline__ void fill_stage_twiddles(V2<T>* tws, const V2<T>* __restrict__ tw) {
  if constexpr (S < plan_nstages<PLAN16>(N)) {
    constexpr int R = plan_radix<PLAN16>(N, S), P = plan_pprod<PLAN16>(N, S);
    constexpr int OFF = tw_offset<PLAN16>(N, S), STEP = TWN / (P * R);
    for (int e = threadIdx.x; e < (R - 1) * P; e += NTH) {
      const int r = e / P + 1, k = e % P;
      tws[OFF + e] = tw[r * k * STEP];
    }
    fill_stage_twiddles<T, N, PLAN16, NTH, S + 1>(tws, tw);
  }
}

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

template <bool INV, typename V> struct DFT<16, INV, V> {
  // n = 4 n1 + n2, k = k1 + 4 k2: DFT4 over n1, twiddle W16^{n2 k1}, DFT4 over n2.
  static __device__ __forceinline__ void run(V* v) {
    using T = decltype(v[0].x);
    const T c1 = T(0.92387953251128675612818318939678828682);  // cos(pi/8)
    const T s1 = T(0.38268343236508977172845998403039886676);  // sin(pi/8)
    const T h = T(0.70710678118654752440084436210484903928);   // sqrt(2)/2
    const T sg = INV ? T(1) : T(-1);                            // sign of the exponent
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) dft4<INV>(v[n2], v[4 + n2], v[8 + n2], v[12 + n2]);
    // element (k1, n2) now sits at v[4*k1 + n2]; twiddle by exp(sg 2 pi i n2 k1 / 16)
    auto tw = [&](V a, T c, T s) {  // a * (c + i sg s)
      V r;
      r.x = a.x * c - sg * a.y * s;
      r.y = a.y * c + sg * a.x * s;
      return r;
    };
    v[5] = tw(v[5], c1, s1);                   // W^1
    v[6] = tw(v[6], h, h);                     // W^2
    v[7] = tw(v[7], s1, c1);                   // W^3
    v[9] = tw(v[9], h, h);                     // W^2
    v[10] = INV ? cmul_i(v[10]) : cmul_mi(v[10]);  // W^4
    v[11] = tw(v[11], -h, h);                  // W^6
    v[13] = tw(v[13], s1, c1);                 // W^3
    v[14] = tw(v[14], -h, h);                  // W^6
    v[15] = tw(v[15], -c1, -s1);               // W^9
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) dft4<INV>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    // X[k1 + 4 k2] is at v[4*k1 + k2]: transpose to natural order
    V t[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) t[i] = v[i];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
      for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[4 * k1 + k2];
  }
};

struct NoHook {
  __device__ void operator()() const {}
};

// Column-tile slot of (pos, col) for W-wide rows, with one pad row after every
// 8 rows.  For every stage of the radix plan, at(b + r*NB) and at(j + r*P) lie
// at offsets from at(b) and at(j) that depend on r alone (step(r*NB) when NB
// is a multiple of 8, step(r*P) always), so a thread addresses all its
// butterfly inputs and outputs from one base slot; and the stride-R rows of the
// first-stage stores of a warp alternate between the two halves of the banks.
template <int W> struct Skew8 {
  static __host__ __device__ constexpr int rows(int N) { return N + (N >> 3); }
  static __device__ __forceinline__ int at(int pos, int col) { return (pos + (pos >> 3)) * W + col; }
  static __host__ __device__ constexpr int step(int d) { return (d + (d >> 3)) * W; }
};
// Slots of one Skew8 buffer of N-row, W-wide tiles.
__host__ __device__ constexpr int skew8_slots(int N, int W) { return (N + (N >> 3)) * W; }

// One Stockham stage.  SRC/DST: 0 = functor, 1 = buffer A, 2 = buffer B.
template <typename T, int N, int NCOLS, int NT, class ADDR, bool INV, int R, int P, int TWO, int SRC, int DST,
          class LD, class ST>
__device__ __forceinline__ void fft_stage_io(V2<T>* __restrict__ A, V2<T>* __restrict__ B,
                                             const V2<T>* __restrict__ tws, LD& ld, ST& st) {
  constexpr int NB = N / R;
  constexpr int TOTAL = NB * NCOLS;
  constexpr int CNT = (TOTAL + NT - 1) / NT;
  const V2<T>* src = SRC == 1 ? A : B;
  V2<T>* dst = DST == 1 ? A : B;
#pragma unroll
  for (int c = 0; c < CNT; ++c) {
    const int t = threadIdx.x + c * NT;
    if (TOTAL % NT == 0 || t < TOTAL) {
      const int col = t % NCOLS, b = t / NCOLS;
      V2<T> v[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if constexpr (SRC == 0) {
          if constexpr (std::is_invocable<LD&, int, int, int, int>::value) v[r] = ld(b + r * NB, col, r, c);
          else if constexpr (std::is_invocable<LD&, int, int, int>::value) v[r] = ld(b + r * NB, col, r);
          else v[r] = ld(b + r * NB, col);
        } else if constexpr (NB % 8 == 0) {
          v[r] = src[ADDR::at(b, col) + ADDR::step(r * NB)];
        } else {
          v[r] = src[ADDR::at(b + r * NB, col)];
        }
      }
      const int k = b & (P - 1);
      if (P > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          V2<T> w = tws[TWO + (r - 1) * P + k];
          if (INV) w.y = -w.y;
          v[r] = cmul(v[r], w);
        }
      }
      DFT<R, INV, V2<T>>::run(v);
      const int j = (b - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if constexpr (DST == 0) {
          if constexpr (std::is_invocable<ST&, int, int, V2<T>, int, int>::value) st(j + r * P, col, v[r], r, c);
          else if constexpr (std::is_invocable<ST&, int, int, V2<T>, int>::value) st(j + r * P, col, v[r], r);
          else st(j + r * P, col, v[r]);
        } else {
          dst[ADDR::at(j, col) + ADDR::step(r * P)] = v[r];
        }
      }
    }
  }
  if (DST != 0) __syncthreads();
}

template <typename T, int N, int NCOLS, int NT, class ADDR, bool INV, int S, class LD, class ST, class HK>
__device__ __forceinline__ void fft_stages_io(V2<T>* A, V2<T>* B, const V2<T>* tws, LD& ld, ST& st, HK& hk) {
  constexpr int NS = fft_nstages(N);
  if constexpr (S < NS) {
    constexpr int SRC = S == 0 ? 0 : ((S - 1) % 2 == 0 ? 1 : 2);
    constexpr int DST = S == NS - 1 ? 0 : (S % 2 == 0 ? 1 : 2);
    fft_stage_io<T, N, NCOLS, NT, ADDR, INV, fft_radix(N, S), fft_pprod(N, S), tw_offset<false>(N, S), SRC, DST>(
        A, B, tws, ld, st);
    if constexpr (S == 0 && !std::is_same<HK, NoHook>::value) {
      if constexpr (DST == 0) __syncthreads();
      hk();
    }
    fft_stages_io<T, N, NCOLS, NT, ADDR, INV, S + 1>(A, B, tws, ld, st, hk);
  }
}

// Unnormalised FFT of NCOLS sequences of length N: inputs from ld(pos, col),
// outputs to st(pos, col, v), intermediate stages in A/B (ADDR::rows(N)*NCOLS
// slots each, slot ADDR::at(pos, col)), twiddles from the shared stage tables
// tws (fill_stage_twiddles<T, N, false>).  INV selects exp(+2 pi i nk/N).  A
// thread's butterflies are t = threadIdx.x + c*NT (col = t % NCOLS, b = t /
// NCOLS); ld may take a third argument r and st a fourth, the index of the
// value within the butterfly (position b + r*N/R in the first stage, j + r*P
// in the last), and ld a fourth and st a fifth, the thread's butterfly index
// c, so a caller can keep a thread's inputs or outputs in registers.  The caller synchronises before ld reads shared memory written by
// other threads and after st writes shared memory that other threads read.
// after_stage0() (optional) runs once every thread has finished the first
// stage, when the loader's source may be reused.
template <typename T, int N, int NCOLS, int NT, class ADDR, bool INV, class LD, class ST, class HK = NoHook>
__device__ __forceinline__ void fft_io(V2<T>* A, V2<T>* B, const V2<T>* tws, LD&& ld, ST&& st,
                                       HK&& after_stage0 = HK{}) {
  static_assert((N & (N - 1)) == 0 && N >= 2 && N <= TWN, "power-of-two length");
  fft_stages_io<T, N, NCOLS, NT, ADDR, INV, 0>(A, B, tws, ld, st, after_stage0);
}
// column tiles of W contiguous columns
template <int N, int W> using TileAddr = Skew8<W>;

// ---------------------------------------------------------------------------
// In-place variant for row FFTs: one shared buffer; each stage loads all of a
// thread's butterfly inputs into registers, the block synchronises, then the
// outputs are written back in place.  Threads map to butterflies with the
// position index fastest (consecutive lanes walk consecutive positions, so a
// loader or storer on global rows coalesces).  ADDR::at(pos, col) gives the
// shared-memory slot (see SkewAddr).
// ---------------------------------------------------------------------------

// Slot of (pos, col): one skew slot every 16 positions keeps the strided
// first-stage stores of the radix plans conflict-free.
template <int LDC> struct SkewAddr {
  static constexpr int LD = LDC;  // slots per column
  static __device__ __forceinline__ int at(int pos, int col) { return col * LD + pos + (pos >> 4); }
};
__host__ __device__ constexpr int skew_ld(int N) { return N + (N >> 4); }

template <typename T, int N, int NCOLS, int NT, class ADDR, bool INV, int R, int P, int TWO, bool FIRST, bool LAST,
          class LD, class ST, class HK>
__device__ __forceinline__ void fft_ip_stage(V2<T>* __restrict__ buf, const V2<T>* __restrict__ tws, LD& ld,
                                             ST& st, HK& after_loads) {
  constexpr int NB = N / R;
  constexpr int TOTAL = NB * NCOLS;
  constexpr int CNT = (TOTAL + NT - 1) / NT;
  V2<T> v[CNT][R];
#pragma unroll
  for (int c = 0; c < CNT; ++c) {
    const int t = threadIdx.x + c * NT;
    if (TOTAL % NT == 0 || t < TOTAL) {
      const int b = t % NB, col = t / NB;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if constexpr (FIRST) v[c][r] = ld(b + r * NB, col);
        else v[c][r] = buf[ADDR::at(b + r * NB, col)];
      }
    }
  }
  __syncthreads();
  if constexpr (FIRST) after_loads();
#pragma unroll
  for (int c = 0; c < CNT; ++c) {
    const int t = threadIdx.x + c * NT;
    if (TOTAL % NT == 0 || t < TOTAL) {
      const int b = t % NB, col = t / NB;
      const int k = b & (P - 1);
      if (P > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          V2<T> w = tws[TWO + (r - 1) * P + k];
          if (INV) w.y = -w.y;
          v[c][r] = cmul(v[c][r], w);
        }
      }
      DFT<R, INV, V2<T>>::run(v[c]);
      const int j = (b - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if constexpr (LAST) st(j + r * P, col, v[c][r]);
        else buf[ADDR::at(j + r * P, col)] = v[c][r];
      }
    }
  }
  __syncthreads();
}

template <typename T, int N, int NCOLS, int NT, class ADDR, bool INV, int S, class LD, class ST, class HK>
__device__ __forceinline__ void fft_ip_stages(V2<T>* buf, const V2<T>* tws, LD& ld, ST& st, HK& hk) {
  constexpr int NS = fft16_nstages(N);
  if constexpr (S < NS) {
    fft_ip_stage<T, N, NCOLS, NT, ADDR, INV, fft16_radix(N, S), fft16_pprod(N, S), tw_offset<true>(N, S), S == 0,
                 S == NS - 1>(buf, tws, ld, st, hk);
    fft_ip_stages<T, N, NCOLS, NT, ADDR, INV, S + 1>(buf, tws, ld, st, hk);
  }
}

// In-place FFT of NCOLS sequences of length N: stage 0 reads ld(pos, col)
// (which may read buf: every thread finishes loading before any store), the
// last stage calls st(pos, col, v) (which may write buf).  Radix-16 plan,
// twiddles from the shared stage tables tws (fill_stage_twiddles<T, N, true>).
// Returns with the block synchronised.
// after_loads() runs once, right after every thread has loaded the inputs of
// the first stage (the loader's source is then free for reuse).
template <typename T, int N, int NCOLS, int NT, class ADDR, bool INV, class LD, class ST, class HK = NoHook>
__device__ __forceinline__ void fft_ip(V2<T>* buf, const V2<T>* tws, LD&& ld, ST&& st, HK&& after_loads = HK{}) {
  static_assert((N & (N - 1)) == 0 && N >= 2 && N <= TWN, "power-of-two length");
  fft_ip_stages<T, N, NCOLS, NT, ADDR, INV, 0>(buf, tws, ld, st, after_loads);
}

// Asynchronous 16-byte global -> shared copies (cp.async, completion tracked
// per thread with commit/wait groups).
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
// TMA bulk prefetch of [gmem, gmem+bytes) into L2 (16-byte aligned, bytes a
// multiple of 16); no completion to wait for.
__device__ __forceinline__ void prefetch_l2(const void* gmem, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// wait until at most N of this thread's most recent cp.async groups are pending
template <int N> __device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

}  // namespace hit
