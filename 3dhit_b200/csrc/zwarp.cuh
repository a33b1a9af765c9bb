// Warp-resident transforms of the fused z pass (float32, H = Nz/2 in {32, 64,
// 128, 256, 512}).
//
// For H <= 256 a warp owns ROWS = 256/H whole (x, y) rows; LPR = H/8 lanes
// serve one row.  For H = 512 a row needs LPR = 64 lanes: a team of two warps
// owns it, and the team's exchanges are ordered by a named barrier over its 64
// threads instead of __syncwarp (zw_sync).
// The half-length complex transform of a row (H points, see k_z.cu) runs on
// the plan radix 8 -> R1 -> radix 8 (R1 = H/64; H = 64 has no middle stage;
// H = 32 is radix 8 -> radix 4 with two radix-4 butterflies per lane):
// every stage leaves each lane holding 8 complex values, the radix-8 stages
// one butterfly per lane, the middle stage 8/R1 butterflies per lane.  Values
// move between stages through a row-private shared exchange buffer, laid out
// so that every access of a half warp hits 16 distinct bank pairs (zw_slot;
// the one exception is the middle stage's stores at H = 128, two-way on some
// pairs), and ordered by __syncwarp (or the team barrier): no CTA barrier
// anywhere in the row loop.
//
// The first stage of the plan reads positions b + (H/8) r of the lane's row
// (b = lane % LPR, r = 0..7) and the last stage writes positions b + (H/8) r,
// so the inverse transforms leave each lane with the same 8 physical positions
// of all six fields: the cross product u x w is formed in registers, and the
// product is already laid out as the forward transform's first-stage input.
// The r2c post-processing pairs Z[k] with Z[H-k], which sits in lane
// (LPR - b) mod LPR of the same row: one __shfl_sync per value (H <= 256), or
// a trip through the exchange buffer when the partner is in the other warp of
// the team (H = 512).
#pragma once

#include "fft_core.cuh"

namespace hit {

template <int H> struct ZW {
  static_assert(H == 32 || H == 64 || H == 128 || H == 256 || H == 512,
                "warp-resident z rows need H in {32, ..., 512}");
  static constexpr int LPR = H / 8;                 // lanes per row
  static constexpr int TEAM = H <= 256 ? 1 : 2;     // warps per row
  static constexpr int ROWS = H <= 256 ? 32 / LPR : 1;  // rows per warp (per team of two at H = 512)
  static constexpr int R1 = H / 64;      // middle radix (1: no middle stage)
  static constexpr int NB0 = H / 8;      // butterflies of a radix-8 stage
  static constexpr int XS = H <= 64 ? H + H / 8 : H + H / 16;  // exchange slots per row (see zw_slot)
  // last stage: radix LR over stride LP (H = 32: two radix-4 butterflies per
  // lane over P = 8; else one radix-8 butterfly per lane over P = H/8)
  static constexpr int LR = H == 32 ? 4 : 8;
  static constexpr int LP = H / LR;
  // twiddle tables: middle stage (R1-1) x 8, last stage (LR-1) x LP, then
  // exp(-2 pi i k / 2H) for k = 0..H (pre/post-processing of the real rows)
  static constexpr int TW1 = 0;
  static constexpr int TW2 = R1 > 1 ? (R1 - 1) * 8 : 0;
  static constexpr int TWZ = TW2 + (LR - 1) * LP;
  static constexpr int TWS = (TWZ + H + 1 + 1) / 2 * 2;  // even: what follows stays 16-byte aligned
};

// Exchange slot of row position p: one pad slot after every 8 positions (H =
// 32, 64) or every 16 (H = 128, 256, 512).  The accesses are, per half warp:
// the first stage's stores of positions 8b + r (16 consecutive b), the middle
// stage's loads of contiguous runs and stores of two runs of 8 positions, the
// last stage's loads of contiguous runs.  An 8-byte slot s uses the bank pair
// of s mod 16, and all of these accesses get 16 distinct pairs except the
// middle stage's stores with butterflies assigned in order (b1 = b + LPR i):
// the tables below fix that at H = 256 and 512; at H = 128 the stores' pairs
// take only 15 values over the 64 butterflies, so some stay two-way.  The
// padding is additive in the fields of p that a lane's index and a value's
// index r fill, so every access is the lane's base slot plus a constant
// offset.
template <int H> __device__ __forceinline__ int zw_slot(int p) {
  return H <= 64 ? p + (p >> 3) : p + (p >> 4);
}

// Twiddle tables of ZW<H> from the global exp(-2 pi i m / TWN) table (all
// threads of the CTA call; the caller synchronises before use).
template <int H, int NTH> __device__ __forceinline__ void zw_fill_twiddles(float2* tws, const float2* __restrict__ tw) {
  using Z = ZW<H>;
  for (int e = threadIdx.x; e < Z::TWS; e += NTH) {
    int m = 0;
    if (e < Z::TW2) {  // middle stage: P = 8, radix R1: w_{8 R1}^{r k}
      const int r = e / 8 + 1, k = e % 8;
      m = r * k * (TWN / (8 * Z::R1));
    } else if (e < Z::TWZ) {  // last stage: P = LP, radix LR: w_H^{r k}
      const int r = (e - Z::TW2) / Z::LP + 1, k = (e - Z::TW2) % Z::LP;
      m = r * k * (TWN / H);
    } else if (e - Z::TWZ <= H) {
      m = (e - Z::TWZ) * (TWN / (2 * H));
    }
    tws[e] = tw[m];
  }
}

// Middle-stage butterflies of a lane (H = 128, 256: C1 = 8 / R1 per lane).
// With the plain assignment b1 = b + LPR i, the stores j + 8 r (j = 32
// (b1 / 8) + b1 % 8) of a half warp at H = 256 put two lanes on 6 of the 8
// bank pairs they use.  The table below assigns the 64 butterflies of H = 256
// to (lane, i) so that every middle-stage load (b1 + 64 r) and store of a half
// warp hits 16 distinct bank pairs under zw_slot: each half warp's 16
// butterflies are one perfect matching of the bipartite graph joining a
// butterfly's load bank pair to its store bank pair (4-regular, so four
// matchings cover it).  Entry [32 i + lane].
__device__ const unsigned char kZwMid256[64] = {
    0, 1,  2,  3,  4,  5,  6,  13, 14, 15, 37, 38, 39, 40, 41, 42, 8,  9,  10, 17, 18, 19,
    20, 21, 28, 29, 30, 31, 47, 52, 56, 57, 7,  11, 12, 16, 32, 33, 34, 35, 36, 43, 44, 45,
    46, 53, 54, 55, 22, 23, 24, 25, 26, 27, 48, 49, 50, 51, 58, 59, 60, 61, 62, 63};

// Orders the exchange-buffer accesses of the threads that share a row: the
// warp for H <= 256, the team's two warps (named barrier `id`, 64 threads) for
// H = 512.
template <int H> __device__ __forceinline__ void zw_sync(int id) {
  if constexpr (ZW<H>::TEAM == 1) {
    __syncwarp();
  } else {
    asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory");
  }
}

// H = 512 (one radix-8 middle butterfly per lane of a two-warp team): with
// b1 = b the stores j + 8 r (j = 64 (b1 / 8) + b1 % 8) of a half warp put two
// lanes on 4 of the bank pairs.  The same construction as for H = 256 -- four
// perfect matchings of the 4-regular bipartite graph joining load bank pair
// (b1 + b1 / 16) mod 16 to store bank pair (b1 % 8 + 4 (b1 / 8)) mod 16 --
// gives each half warp of the team 16 butterflies whose loads and stores all
// hit distinct bank pairs.  Entry [team lane].
__device__ const unsigned char kZwMid512[64] = {
    0,  1,  2,  3,  4,  9,  10, 11, 12, 13, 14, 15, 20, 21, 22, 23, 5,  6,  7,  8,  16, 17,
    18, 19, 24, 25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 41, 42, 43, 44, 45, 46, 47,
    52, 53, 54, 55, 37, 38, 39, 40, 48, 49, 50, 51, 56, 57, 58, 59, 60, 61, 62, 63};

template <int H> struct ZwMid {
  static constexpr int R1 = ZW<H>::R1, C1 = R1 > 1 ? 8 / R1 : 1;
  int k[C1];   // twiddle index b1 % 8
  int ld[C1];  // exchange slot of input b1 (input r at ld + zw_slot(r H / R1))
  int st[C1];  // exchange slot of output j (output r at st + zw_slot(8 r))
  // once per thread (a load of the table at H = 256, 512).  The offsets are
  // additive: H / R1 = 64 is a multiple of 16, and j % 16 = b1 % 8 leaves
  // room for 8 r % 16 below 16.
  __device__ __forceinline__ explicit ZwMid(int b) {
#pragma unroll
    for (int i = 0; i < C1; ++i) {
      const int b1 = H == 256   ? (int)kZwMid256[32 * i + b]
                     : H == 512 ? (int)kZwMid512[b]
                                : b + ZW<H>::LPR * i;
      k[i] = b1 & 7;
      ld[i] = zw_slot<H>(b1);
      st[i] = zw_slot<H>((b1 - k[i]) * R1 + k[i]);
    }
  }
};

// The three stages of one H-point transform (INV: exp(+2 pi i nk/H)).  On
// entry v[r] holds position b + (H/8) r of the lane's row, on exit output
// b + (H/8) r.  xch is the row's exchange buffer; mid the lane's middle-stage
// butterflies; the warp (the team at H = 512, barrier bar_id) must call this
// converged.  Returns with the exchange buffer free for the next transform.
template <int H, bool INV>
__device__ __forceinline__ void zw_transform(float2 (&v)[8], float2* xch, const float2* __restrict__ tws, int b,
                                             const ZwMid<H>& mid, const float2 (&wl)[7], int bar_id = 0) {
  using Z = ZW<H>;
  if constexpr (H == 32) {
    // 8 x 4: stage 0 as below, then two radix-4 butterflies j = b + 4h (P = 8,
    // inputs and outputs j + 8r), whose outputs b + 4 (h + 2r) are the lane's
    // positions b + (H/8) r' with r' = h + 2r
    DFT<8, INV, float2>::run(v);
#pragma unroll
    for (int r = 0; r < 8; ++r) xch[zw_slot<H>(8 * b + r)] = v[r];
    zw_sync<H>(bar_id);
    float2 u[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
#pragma unroll
      for (int r = 0; r < 4; ++r) u[h][r] = xch[zw_slot<H>(b + 4 * h + 8 * r)];
    }
    zw_sync<H>(bar_id);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
#pragma unroll
      for (int r = 1; r < 4; ++r) {
        float2 w = wl[3 * h + r - 1];
        if (INV) w.y = -w.y;
        u[h][r] = cmul(u[h][r], w);
      }
      DFT<4, INV, float2>::run(u[h]);
#pragma unroll
      for (int r = 0; r < 4; ++r) v[h + 2 * r] = u[h][r];
    }
    return;
  }
  DFT<8, INV, float2>::run(v);  // stage 0 (P = 1): outputs 8b + r
#pragma unroll
  for (int r = 0; r < 8; ++r) xch[zw_slot<H>(8 * b + r)] = v[r];
  zw_sync<H>(bar_id);
  if constexpr (Z::R1 > 1) {
    constexpr int R1 = Z::R1, NB1 = H / R1, C1 = 8 / R1;
    float2 u[C1][R1];
    static_assert(NB1 % 16 == 0, "additive exchange offsets");
#pragma unroll
    for (int i = 0; i < C1; ++i) {
#pragma unroll
      for (int r = 0; r < R1; ++r) u[i][r] = xch[mid.ld[i] + zw_slot<H>(NB1 * r)];
    }
    zw_sync<H>(bar_id);
#pragma unroll
    for (int i = 0; i < C1; ++i) {
      const int k = mid.k[i];
#pragma unroll
      for (int r = 1; r < R1; ++r) {
        float2 w = tws[Z::TW1 + (r - 1) * 8 + k];
        if (INV) w.y = -w.y;
        u[i][r] = cmul(u[i][r], w);
      }
      DFT<R1, INV, float2>::run(u[i]);
#pragma unroll
      for (int r = 0; r < R1; ++r) xch[mid.st[i] + zw_slot<H>(8 * r)] = u[i][r];
    }
    zw_sync<H>(bar_id);
  }
  // last stage: radix 8, P = H/8, butterfly b (k = b, outputs b + (H/8) r)
#pragma unroll
  for (int r = 0; r < 8; ++r) v[r] = xch[zw_slot<H>(b + Z::NB0 * r)];
  zw_sync<H>(bar_id);
#pragma unroll
  for (int r = 1; r < 8; ++r) {
    float2 w = wl[r - 1];
    if (INV) w.y = -w.y;
    v[r] = cmul(v[r], w);
  }
  DFT<8, INV, float2>::run(v);
}

// The last stage's twiddles w_H^{r b}, r = 1..7, of lane b: the same for every
// row and transform the lane handles, so they are loaded once into registers
// (the shared-memory loads they replace were an eighth of a row's exchange
// traffic).
template <int H> __device__ __forceinline__ void zw_last_twiddles(float2 (&wl)[7], const float2* tws, int b) {
  using Z = ZW<H>;
  if constexpr (H == 32) {  // w_32^{r j}, j = b + 4h, at wl[3h + r - 1]
#pragma unroll
    for (int h = 0; h < 2; ++h) {
#pragma unroll
      for (int r = 1; r < 4; ++r) wl[3 * h + r - 1] = tws[Z::TW2 + (r - 1) * Z::LP + b + 4 * h];
    }
    wl[6] = make_float2(1.f, 0.f);
  } else {
#pragma unroll
    for (int r = 1; r < 8; ++r) wl[r - 1] = tws[Z::TW2 + (r - 1) * Z::NB0 + b];
  }
}

// e^{-2 pi i k / (2H)} at k = b + (H/8) r from w0 = e^{-2 pi i b / (2H)}: the
// step (H/8)/(2H) = 1/16 of a turn is the same for every H, so the factor is
// w0 times e^{-i pi r / 8} (exact for r = 0 and 4).  This keeps one complex
// value per lane instead of eight.  Called in fully unrolled loops, where r is
// a constant and the selection folds away.
__device__ __forceinline__ float2 zw_wz(float2 w0, int r) {
  constexpr float c = 0.92387953251128675613f, s = 0.38268343236508977173f, h = 0.70710678118654752440f;
  if (r == 0) return w0;
  if (r == 4) return make_float2(w0.y, -w0.x);
  const float cr = r == 1 ? c : r == 2 ? h : r == 3 ? s : r == 5 ? -s : r == 6 ? -h : -c;
  const float ci = r == 1 ? -s : r == 2 ? -h : r == 3 ? -c : r == 5 ? -c : r == 6 ? -h : -s;
  return cmul(w0, make_float2(cr, ci));
}

}  // namespace hit
