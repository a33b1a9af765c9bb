// Column FFT kernels along the strided spectral axes (x and y).
//
// A CTA owns one tile: all N positions along the transformed axis times W
// contiguous z columns, for one value of the remaining axis.  Rows along the
// axis are "compact" (see Geom): rows that are not stored are zeros on input
// and dropped on output, so the dealiased path never moves the 5/9 of the
// x/y frequencies the 2/3 rule removes.  The first FFT stage reads straight
// from global memory (or from the fused prologue) and the last stage writes
// straight to global memory (or to the fused epilogue); only the middle stages
// go through shared memory.
//
// k_p1 and k_p3 are the x-axis ends of the RHS (src/hit3d/navierstokes.py:69-95):
//   k_p1: curl (navierstokes.py:73-77) and the x part of to_physical for u and w;
//   k_p3: x part of to_spectral, forcing (forcing.py:94-95,138-143), dealias +
//         projection (grid.py:166-178), viscous term (navierstokes.py:95) and
//         the RK4 stage algebra (integrators.py:32-38), then -- fused -- the
//         next stage's k_p1 on the tile it just produced.
#include <algorithm>
#include <cstdint>
#include <type_traits>

#include "fft_core.cuh"
#include "kernels.h"
#include "tc_common.cuh"
#include "tma.cuh"

namespace hit {

// Position of a persistent block's tile in the decomposition
// tile = (c * no + o) * nzt + zt, advanced by the grid stride with carries
// (the stride is decomposed once) instead of dividing every tile index.
struct TileWalk {
  int zt, o, c, dz, dq, dc, nzt, no;
  __device__ __forceinline__ TileWalk(int t, int stride, int nzt_, int no_) : nzt(nzt_), no(no_) {
    zt = t % nzt;
    o = (t / nzt) % no;
    c = (t / nzt) / no;
    dz = stride % nzt;
    dq = (stride / nzt) % no;
    dc = (stride / nzt) / no;
  }
  __device__ __forceinline__ TileWalk next() const {
    TileWalk w = *this;
    w.zt += dz;
    int cy = w.zt >= nzt;
    if (cy) w.zt -= nzt;
    w.o += dq + cy;
    cy = w.o >= no;
    if (cy) w.o -= no;
    w.c += dc + cy;
    return w;
  }
};

// PF (staging mode): 0 = the first stage reads global memory directly;
// 1 = the next tile's stored rows are staged in shared memory with cp.async
// while the current tile is transformed (16-byte aligned rows, whole tiles
// inside the source rows); 2 = the same staging with TMA: one thread loads the
// tile as boxes of br rows x W columns through two tensor maps, one over the
// stored rows [0, hin) (to positions [0, ka*br)) and one over [hin, Min) (to
// positions [N - kb*br, N), the boxes aligned to the end of that half); rows
// of a box outside its half are zero-filled by the TMA unit and land in the
// gap between the halves.  The staging buffer holds all N positions: rows that
// are never loaded stay zero from the kernel start, so the first stage reads it
// without checks.  The inverse transform always writes all N rows and the
// forward one always reads all N rows (the launcher checks this).
constexpr int AXIS_WAIT = 1 << 22;  // mbarrier polls before a TMA wait gives up
__device__ int g_axis_timeout = 0;  // set when a TMA wait gave up (hit_device_status)
// Polls of the wait for a tile's boxes (hit_set_wait_limit lowers it so that
// a test can make the wait give up); the wait for the copies still in flight
// after a give-up always polls AXIS_WAIT times.
__device__ int g_axis_wait_limit = AXIS_WAIT;

template <typename T, int N, int W, bool INV, int PF>
__global__ void __launch_bounds__(NT) k_axis(AxisArgs<T> a, int nzt, int no, int ntiles,
                                             const __grid_constant__ CUtensorMap mapA,
                                             const __grid_constant__ CUtensorMap mapB) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t tbar;
  V2<T>* A = reinterpret_cast<V2<T>*>(smem_raw);
  V2<T>* B = A + skew8_slots(N, W);
  V2<T>* tws = B + skew8_slots(N, W);
  // N x W staged rows, 128-byte aligned (TMA destinations)
  V2<T>* stg = reinterpret_cast<V2<T>*>(
      (reinterpret_cast<uintptr_t>(tws + ((tw_size<false>(N) + 1) / 2 * 2)) + 127) & ~(uintptr_t)127);
  fill_stage_twiddles<T, N, false, NT>(tws, a.tw);
  constexpr int VPC = 16 / sizeof(V2<T>);
  constexpr int XE = sizeof(V2<T>) / 8;  // 8-byte tensor elements per complex value
  const uint32_t mb = tma::smem_u32(&tbar);
  auto prefetch = [&](const TileWalk& w) {
    if constexpr (PF == 1) {
      const V2<T>* src = a.src + w.c * a.s_c + w.o * a.s_o + w.zt * W;
      constexpr int CPR = W / VPC;  // 16-byte chunks per row
      for (int e = threadIdx.x; e < a.Min * CPR; e += NT) {
        const int row = e / CPR, ch = e % CPR;
        cp_async16(stg + full_pos(row, a.hin, a.Min, N) * W + ch * VPC, src + (long long)row * a.s_a + ch * VPC);
      }
      cp_async_commit();
    } else if constexpr (PF == 2) {
      if (threadIdx.x == 0) {
        tma::mbar_expect_tx(mb, (uint32_t)((a.ka + a.kb) * a.br * W * sizeof(V2<T>)));
        const int x = w.zt * W * XE;
        for (int k = 0; k < a.ka; ++k) tma::load4(stg + k * a.br * W, &mapA, x, k * a.br, w.o, w.c, mb);
        for (int k = 0; k < a.kb; ++k)
          tma::load4(stg + (N - (k + 1) * a.br) * W, &mapB, x, a.pb - (k + 1) * a.br, w.o, w.c, mb);
      }
    }
  };
  if constexpr (PF == 1) {
    for (int e = threadIdx.x; e < (N - a.Min) * W; e += NT) stg[a.hin * W + e] = czero<T>();
  } else if constexpr (PF == 2) {
    for (int e = threadIdx.x; e < (N - (a.ka + a.kb) * a.br) * W; e += NT) stg[a.ka * a.br * W + e] = czero<T>();
    if (threadIdx.x == 0) tma::mbar_init(mb, 1);
    tma::fence_async_smem();
  }
  TileWalk walk(blockIdx.x, gridDim.x, nzt, no);
  const int wait_limit = PF == 2 ? g_axis_wait_limit : 0;
  pdl_wait();
  pdl_trigger();
  __syncthreads();
  if (PF != 0 && blockIdx.x < ntiles) prefetch(walk);
  if constexpr (PF != 2) __syncthreads();
  uint32_t phase = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int z0 = walk.zt * W;
    const long long o = walk.o, c = walk.c;
    const V2<T>* src = a.src + c * a.s_c + o * a.s_o + z0;
    V2<T>* dst = a.dst + c * a.d_c + o * a.d_o + z0;
    const bool zc = z0 + W <= a.nz;  // whole tile inside the valid columns
    if constexpr (PF == 1) {
      cp_async_wait_all();
      __syncthreads();
    } else if constexpr (PF == 2) {
      // the tile's boxes have landed (a verdict shared by the block)
      const bool ok = __syncthreads_and(tma::mbar_wait(mb, phase, wait_limit)) != 0;
      phase ^= 1;
      if (!ok) {
        if (threadIdx.x == 0) atomicExch(&g_axis_timeout, 1);
        tma::mbar_wait(mb, phase ^ 1, AXIS_WAIT);  // the copies in flight, once more with a limit
        return;
      }
    }
    const int nxt = tile + gridDim.x;
    const TileWalk nwalk = walk.next();
    fft_io<T, N, W, NT, TileAddr<N, W>, INV>(
        A, B, tws,
        [&](int pos, int col) {
          if (PF != 0) return stg[pos * W + col];
          const int row = INV ? compact_row(pos, a.hin, a.Min, N) : pos;
          return (row >= 0 && (zc || z0 + col < a.nz)) ? src[(long long)row * a.s_a + col] : czero<T>();
        },
        [&](int pos, int col, V2<T> v) {
          const int row = INV ? pos : compact_row(pos, a.hout, a.Mout, N);
          if (row >= 0 && (zc || z0 + col < a.nz)) dst[(long long)row * a.d_a + col] = v;
        },
        [&]() {
          if (PF != 0 && nxt < ntiles) prefetch(nwalk);
        });
    __syncthreads();  // the next tile's first stage rewrites A
    walk = nwalk;
  }
  if constexpr (PF == 1) cp_async_wait_all();
}

// x-inverse of u and w = i k x u for one (ky row, z tile).  comp(c, pos, col,
// r) gives component c of the stage input at full x position pos (zero where
// the position is not stored); r is the index of pos in the calling thread's
// first-stage butterfly, so a caller may serve it from registers.
//
// The x-inverse is linear and ky, kz are constant along an x column, so of
// w = i (ky u_z - kz u_y, kz u_x - kx u_z, kx u_y - ky u_x)
// (navierstokes.py:73-77) only the kx terms need transforms of their own:
// five transforms (u_x, kx u_y, kx u_z, u_y, u_z) give all six fields, w being
// formed from them at the last stage, where a thread holds the same positions
// of every transform (one transform's outputs are kept in registers).
template <typename T, int N, int W, int NTH, class SRC>
__device__ __forceinline__ void p1_body(SRC&& comp, V2<T>* A, V2<T>* B, int j, int z0, const Geom& g,
                                        const KTab<T>& kt, const V2<T>* tws, V2<T>* t6, long long t_c,
                                        long long t_x) {
  const int fy = full_pos(j, g.hy, g.My, g.Ny);
  const T ky = kt.ky[fy];
  V2<T>* out = t6 + (long long)j * g.Mzp + z0;
  constexpr int NS = fft_nstages(N), RL = fft_radix(N, NS - 1);
  constexpr int CNTL = ((N / RL) * W + NTH - 1) / NTH;  // last-stage butterflies per thread
  V2<T> keep[CNTL][RL];
  auto kz_of = [&](int col) {
    const int z = z0 + col;
    return z < g.Nzh ? kt.kz[z] : T(0);
  };
  auto put = [&](int q, int pos, int col, V2<T> v) { out[q * t_c + (long long)pos * t_x + col] = v; };
  auto sync = [&]() {
    // ping-pong: an even stage count ends reading A, which the next
    // transform's first stage rewrites
    if constexpr (NS % 2 == 0) __syncthreads();
  };
  // u_x (kept)
  fft_io<T, N, W, NTH, TileAddr<N, W>, true>(
      A, B, tws, [&](int pos, int col, int r) { return comp(0, pos, col, r); },
      [&](int pos, int col, V2<T> v, int r, int c) {
        put(0, pos, col, v);
        keep[c][r] = v;
      });
  sync();
  // kx u_y -> w_z = i (X_y - ky u_x)
  fft_io<T, N, W, NTH, TileAddr<N, W>, true>(
      A, B, tws, [&](int pos, int col, int r) { return cscale(comp(1, pos, col, r), kt.kx[pos]); },
      [&](int pos, int col, V2<T> v, int r, int c) { put(5, pos, col, cmul_i(csub(v, cscale(keep[c][r], ky)))); });
  sync();
  // kx u_z -> w_y = i (kz u_x - X_z)
  fft_io<T, N, W, NTH, TileAddr<N, W>, true>(
      A, B, tws, [&](int pos, int col, int r) { return cscale(comp(2, pos, col, r), kt.kx[pos]); },
      [&](int pos, int col, V2<T> v, int r, int c) {
        put(4, pos, col, cmul_i(csub(cscale(keep[c][r], kz_of(col)), v)));
      });
  sync();
  // u_y (kept)
  fft_io<T, N, W, NTH, TileAddr<N, W>, true>(
      A, B, tws, [&](int pos, int col, int r) { return comp(1, pos, col, r); },
      [&](int pos, int col, V2<T> v, int r, int c) {
        put(1, pos, col, v);
        keep[c][r] = v;
      });
  sync();
  // u_z -> w_x = i (ky u_z - kz u_y)
  fft_io<T, N, W, NTH, TileAddr<N, W>, true>(
      A, B, tws, [&](int pos, int col, int r) { return comp(2, pos, col, r); },
      [&](int pos, int col, V2<T> v, int r, int c) {
        put(2, pos, col, v);
        put(3, pos, col, cmul_i(csub(cscale(v, ky), cscale(keep[c][r], kz_of(col)))));
      });
  sync();
}

// x-inverse for the fused LES stage: u and the nine velocity gradients
// g_ij = d_j u_i (spectral i k_j u_i, in the order 3 i + j of
// hit_velocity_gradients) of one (ky row, z tile), 12 outputs (u_x, u_y, u_z,
// g_00 .. g_22).  ky and kz are constant along an x column, so six transforms
// (u_i and kx u_i) give all of them; the z pass forms w from the gradients.
template <typename T, int N, int W, int NTH, class SRC>
__device__ __forceinline__ void p1les_body(SRC&& comp, V2<T>* A, V2<T>* B, int j, int z0, const Geom& g,
                                           const KTab<T>& kt, const V2<T>* tws, V2<T>* t12, long long t_c,
                                           long long t_x) {
  const int fy = full_pos(j, g.hy, g.My, g.Ny);
  const T ky = kt.ky[fy];
  V2<T>* out = t12 + (long long)j * g.Mzp + z0;
  constexpr int NS = fft_nstages(N);
  auto kz_of = [&](int col) {
    const int z = z0 + col;
    return z < g.Nzh ? kt.kz[z] : T(0);
  };
  auto put = [&](int q, int pos, int col, V2<T> v) { out[q * t_c + (long long)pos * t_x + col] = v; };
  auto sync = [&]() {
    if constexpr (NS % 2 == 0) __syncthreads();
  };
#pragma unroll 1
  for (int i = 0; i < 3; ++i) {
    // u_i -> u_i, g_i1 = i ky u_i, g_i2 = i kz u_i
    fft_io<T, N, W, NTH, TileAddr<N, W>, true>(
        A, B, tws, [&](int pos, int col, int r) { return comp(i, pos, col, r); },
        [&](int pos, int col, V2<T> v) {
          put(i, pos, col, v);
          put(3 + 3 * i + 1, pos, col, cmul_i(cscale(v, ky)));
          put(3 + 3 * i + 2, pos, col, cmul_i(cscale(v, kz_of(col))));
        });
    sync();
    // kx u_i -> g_i0
    fft_io<T, N, W, NTH, TileAddr<N, W>, true>(
        A, B, tws, [&](int pos, int col, int r) { return cscale(comp(i, pos, col, r), kt.kx[pos]); },
        [&](int pos, int col, V2<T> v) { put(3 + 3 * i, pos, col, cmul_i(v)); });
    sync();
  }
}

template <typename T, int N, int W, int NTH>
__global__ void __launch_bounds__(NTH) k_p1(P1Args<T> a, int nzt, int ntiles) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const Geom& g = a.g;
  V2<T>* A = reinterpret_cast<V2<T>*>(smem_raw);
  V2<T>* B = A + skew8_slots(N, W);
  V2<T>* tws = B + skew8_slots(N, W);
  V2<T>* S = tws + (tw_size<false>(N) + 1) / 2 * 2;  // 3 x N x W, rows not stored stay zero
  fill_stage_twiddles<T, N, false, NTH>(tws, a.tw);
  constexpr int NW = N * W;
  for (int e = threadIdx.x; e < 3 * (N - g.Mx) * W; e += NTH) {
    const int c = e / ((N - g.Mx) * W), r = e % ((N - g.Mx) * W);
    S[c * NW + g.hx * W + r] = czero<T>();
  }
  pdl_wait();
  pdl_trigger();
  const int MW = g.Mx * W;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int j = tile / nzt, z0 = (tile % nzt) * W;
    const V2<T>* src = a.s + (long long)j * g.Mzp + z0;
    const int nxt = tile + gridDim.x;
    if (nxt < ntiles) {  // next tile's rows into L2 while this one is transformed
      const V2<T>* ns = a.s + (long long)(nxt / nzt) * g.Mzp + (nxt % nzt) * W;
      for (int c = 0; c < 3; ++c)
        for (int i = threadIdx.x; i < g.Mx; i += NTH)
          prefetch_l2(ns + c * a.s_c + (long long)i * a.s_x, W * sizeof(V2<T>));
    }
    __syncthreads();  // the previous tile's transforms have read S
    for (int c = 0; c < 3; ++c)
      for (int e = threadIdx.x; e < MW; e += NTH) {
        const int i = e / W, col = e % W;
        S[c * NW + full_pos(i, g.hx, g.Mx, N) * W + col] = src[c * a.s_c + (long long)i * a.s_x + col];
      }
    __syncthreads();
    if (a.les)
      p1les_body<T, N, W, NTH>([&](int c, int pos, int col, int) { return S[c * NW + pos * W + col]; }, A, B, j, z0,
                               g, a.k, tws, a.t6, a.t_c, a.t_x);
    else
      p1_body<T, N, W, NTH>([&](int c, int pos, int col, int) { return S[c * NW + pos * W + col]; }, A, B, j, z0, g,
                            a.k, tws, a.t6, a.t_c, a.t_x);
  }
}

// Register-resident P3: with radix-8 first and last stages and one butterfly
// per thread of those (N/8 * W == NTH) the forward transform's last stage leaves thread
// (b, col) holding positions b + r*N/8, exactly the inputs its first inverse
// stage needs, so the nonlinear term, the epilogue and the new stage input
// never pass through shared memory.
template <int N, int W, int NTH> __host__ __device__ constexpr bool p3_in_regs() {
  return N >= 64 && fft_radix(N, 0) == 8 && fft_radix(N, fft_nstages(N) - 1) == 8 && (N / 8) * W == NTH;
}
// Instantiations that run the fused LES stage (float32, shared-memory mode,
// columns of at most 256 points): their nl tile holds 3 more components, the
// divergence k_j tau_hat_ij of the SGS stress.
template <typename T, int N, int W, int NTH> __host__ __device__ constexpr bool p3_les() {
  return std::is_same<T, float>::value && !p3_in_regs<N, W, NTH>() && N <= 256;
}

// State rows of one mode for the epilogue: us = stage input (u for stages
// 0/1), ac/uu = accumulator and u (stages 2..4).
template <typename T>
__device__ __forceinline__ void p3_load(const P3Args<T>& a, long long o, V2<T> (&us)[3], V2<T> (&ac)[3],
                                        V2<T> (&uu)[3]) {
  const V2<T>* __restrict__ pus = a.stage <= 1 ? a.u : a.s;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    us[c] = pus[c * a.c_c + o];
    if (a.stage >= 2) {
      ac[c] = a.acc[c * a.c_c + o];
      uu[c] = a.u[c * a.c_c + o];
    }
  }
}

// RHS epilogue of one stored mode (x position pos, z index z, state offset
// o): du holds the x-forward nonlinear term (u x w)^ on entry.  Forcing is
// added before dealias and projection (navierstokes.py:88-92), then the
// viscous term (navierstokes.py:95) and the RK4 stage algebra
// (integrators.py:32-38); ns receives the new stage input (or new state) and
// the float64 partial sums are accumulated.
template <typename T>
__device__ __forceinline__ void p3_point(const P3Args<T>& a, int pos, int fy, int z, T ky, T kz, T cf, long long o,
                                         V2<T> (&du)[3], const V2<T> (&us)[3], const V2<T> (&ac)[3],
                                         const V2<T> (&uu)[3], V2<T> (&ns)[3], double& sE, double& sO,
                                         double& sB) {
  const Geom& g = a.g;
  const T kx = __ldg(a.k.kx + pos);
  const T k2 = k2_of(kx, ky, kz);
  const T ik2 = inv_k2_of(k2);
  if (a.fext) {
#pragma unroll
    for (int c = 0; c < 3; ++c) du[c] = cadd(du[c], a.fext[c * a.c_c + o]);
  }
  if (a.forcing == 1) {
#pragma unroll
    for (int c = 0; c < 3; ++c) du[c] = cadd(du[c], cscale(us[c], a.fA));
  } else if (a.forcing == 2) {
    if (a.kmin2 <= k2 && k2 <= a.kmax2) {
#pragma unroll
      for (int c = 0; c < 3; ++c) du[c] = cadd(du[c], cscale(us[c], cf));
    }
  } else if (a.forcing == 3) {
#pragma unroll
    for (int c = 0; c < 3; ++c) du[c] = cadd(du[c], cscale(us[c], cf));
  }
  // every stored mode of the dealiased path lies inside the 2/3 box
  if (g.pruned ? (pos | fy | z) == 0 : !in_dealias(g, pos, fy, z)) {
    du[0] = du[1] = du[2] = czero<T>();
  }
  // projection: div = (kx d0 + ky d1 + kz d2) / k^2 ; d -= k div
  V2<T> div;
  div.x = (kx * du[0].x + ky * du[1].x + kz * du[2].x) * ik2;
  div.y = (kx * du[0].y + ky * du[1].y + kz * du[2].y) * ik2;
  du[0] = csub(du[0], cscale(div, kx));
  du[1] = csub(du[1], cscale(div, ky));
  du[2] = csub(du[2], cscale(div, kz));
  const T nk2 = a.nu * k2;
#pragma unroll
  for (int c = 0; c < 3; ++c) du[c] = csub(du[c], cscale(us[c], nk2));

  V2<T>* __restrict__ pu = a.u;
  V2<T>* __restrict__ pacc = a.acc;
  V2<T>* __restrict__ ps = a.s;
  V2<T>* __restrict__ pout = a.out;
  if (a.ifrk && a.stage > 0) {
    // integrating-factor (Lawson) RK4 with E = e^{-nu k^2 dt/2} and N the RHS
    // without its viscous term:
    //   s2 = E (u + dt/2 k1),  s3 = E u + dt/2 k2,  s4 = E^2 u + dt E k3,
    //   u' = E^2 u + dt/6 ((E (E k1 + 2 k2) + 2 E k3) + k4)
    // (acc holds E k1, then E (E k1 + 2 k2), then + 2 E k3)
    const T E = visc_factor(a.nuh, k2);
    switch (a.stage) {
      case 1:
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          pacc[c * a.c_c + o] = cscale(du[c], E);
          ns[c] = cscale(cadd(us[c], cscale(du[c], a.a_next)), E);
          ps[c * a.c_c + o] = ns[c];
        }
        break;
      case 2:
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          V2<T> acn = ac[c];
          acn.x = acn.x + T(2) * du[c].x;
          acn.y = acn.y + T(2) * du[c].y;
          pacc[c * a.c_c + o] = cscale(acn, E);
          ns[c] = cadd(cscale(uu[c], E), cscale(du[c], a.a_next));
          ps[c * a.c_c + o] = ns[c];
        }
        break;
      case 3:
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const V2<T> ek = cscale(du[c], E);
          V2<T> acn = ac[c];
          acn.x = acn.x + T(2) * ek.x;
          acn.y = acn.y + T(2) * ek.y;
          pacc[c * a.c_c + o] = acn;
          ns[c] = cadd(cscale(uu[c], E * E), cscale(ek, a.a_next));
          ps[c * a.c_c + o] = ns[c];
        }
        break;
      default:
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const V2<T> acn = cadd(ac[c], du[c]);
          ns[c] = cadd(cscale(uu[c], E * E), cscale(acn, a.dt6));
          pu[c * a.c_c + o] = ns[c];
        }
        break;
    }
  } else switch (a.stage) {
    case 0:
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        pout[c * a.c_c + o] = du[c];
        ns[c] = czero<T>();
      }
      break;
    case 1:
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        pacc[c * a.c_c + o] = du[c];
        ns[c] = cadd(us[c], cscale(du[c], a.a_next));
        ps[c * a.c_c + o] = ns[c];
      }
      break;
    case 2:
    case 3:
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        V2<T> acn = ac[c];
        acn.x = acn.x + T(2) * du[c].x;
        acn.y = acn.y + T(2) * du[c].y;
        pacc[c * a.c_c + o] = acn;
        ns[c] = cadd(uu[c], cscale(du[c], a.a_next));
        ps[c * a.c_c + o] = ns[c];
      }
      break;
    default:
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const V2<T> acn = cadd(ac[c], du[c]);
        ns[c] = cadd(uu[c], cscale(acn, a.dt6));
        pu[c * a.c_c + o] = ns[c];
      }
      break;
  }
  if (a.partial) {
    double a2 = 0.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) a2 += (double)ns[c].x * ns[c].x + (double)ns[c].y * ns[c].y;
    const double w = herm_weight(g, z);
    sE += w * a2;
    sO += w * (double)k2 * a2;
    if (a.kmin2 <= k2 && k2 <= a.kmax2) sB += w * a2;
  }
}

// Register mode: the epilogue runs in 8 passes, pass r over the positions
// r*N/8 .. r*N/8 + N/8 - 1 (position b + r*N/8 of every thread).  The state
// rows of a pass (up to 3 arrays x 3 components x N/8 rows x W) are copied to
// a 3-slot shared-memory ring with cp.async two passes ahead, the first two
// while the last forward transform runs, so the epilogue reads shared memory.
template <int N, int W> constexpr int p3_ring_slot() { return 9 * (N / 8) * W; }

// One (ky row, z tile) of P3.  stg holds the staged first nl component of this
// tile; A/B are the FFT buffers; F holds, in shared-memory mode, the nonlinear
// term and then the new stage input in compact rows (3 x Mx x W), and in
// register mode the epilogue's state ring (3 slots of p3_ring_slot).
template <typename T, int N, int W, int NTH>
__device__ __forceinline__ void p3_tile(const P3Args<T>& a, V2<T>* A, V2<T>* B, const V2<T>* tws, V2<T>* F, double* red,
                                        int j, int z0, int tile, V2<T>* stg, int nzt, int ntiles) {
  constexpr bool REGS = p3_in_regs<N, W, NTH>();
  constexpr bool LES = p3_les<T, N, W, NTH>();
  const Geom& g = a.g;
  const int MW = g.Mx * W;
  constexpr int VPC = 16 / sizeof(V2<T>);
  // staged x column of one nl component (N x W)
  auto prefetch = [&](int t, int c, V2<T>* dstb) {
    const int jj = t / nzt, zz = (t % nzt) * W;
    const V2<T>* src = a.t3 + c * a.t_c + (long long)jj * g.Mzp + zz;
    constexpr int CPR = W / VPC;
    for (int e = threadIdx.x; e < N * CPR; e += NTH) {
      const int row = e / CPR, ch = e % CPR;
      cp_async16(dstb + row * W + ch * VPC, src + (long long)row * a.t_x + ch * VPC);
    }
    cp_async_commit();
  };

  // pull the state rows the epilogue reads into L2 while the forward
  // transforms run (one 16-byte-aligned W-wide row segment per prefetch)
  {
    const int nq = a.stage <= 1 ? 3 : 9;  // (array, component): u | s, acc, u
    const long long cbase = (long long)j * g.Mzp + z0;
    for (int q = 0; q < nq; ++q) {
      const V2<T>* arr = q < 3 ? (a.stage <= 1 ? a.u : a.s) : (q < 6 ? a.acc : a.u);
      const V2<T>* base = arr + (q % 3) * a.c_c + cbase;
      for (int i = threadIdx.x; i < g.Mx; i += NTH) prefetch_l2(base + (long long)i * a.c_x, W * sizeof(V2<T>));
    }
  }

  // register mode: copy the state rows of epilogue pass r into ring slot r % 3
  const V2<T>* __restrict__ us_arr = a.stage <= 1 ? a.u : a.s;
  auto stage_pass = [&](int r) {
    if constexpr (REGS) {
      constexpr int NB = N / 8, CPR = W / VPC;
      const int nq = a.stage <= 1 ? 3 : 9;
      V2<T>* slot = F + (r % 3) * p3_ring_slot<N, W>();
      const long long cbase = (long long)j * g.Mzp + z0;
      for (int e = threadIdx.x; e < nq * NB * CPR; e += NTH) {
        const int q = e / (NB * CPR), rem = e % (NB * CPR), lr = rem / CPR, ch = rem % CPR;
        const int i = compact_row(r * NB + lr, g.hx, g.Mx, N);
        if (i >= 0) {
          const V2<T>* arr = q < 3 ? us_arr : (q < 6 ? a.acc : a.u);
          cp_async16(slot + (q * NB + lr) * W + ch * VPC,
                     arr + (q % 3) * a.c_c + cbase + (long long)i * a.c_x + ch * VPC);
        }
      }
      cp_async_commit();
    }
  };

  // registers of the in-register mode: f[c][r] = component c at position
  // b + r*N/8 of column col (nl, then the new stage input)
  V2<T> f[3][REGS ? 8 : 1];
  const auto nl_store = [&](int c) {
    return [&, c](int pos, int col, V2<T> v, int r) {
      if constexpr (REGS) {
        f[c][r] = v;
      } else {
        const int row = compact_row(pos, g.hx, g.Mx, N);
        if (row >= 0) F[c * MW + row * W + col] = v;
      }
    };
  };
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    cp_async_wait_all();
    __syncthreads();
    // once the first stage has read the staged column, stage the next one:
    // component c+1 of this tile, or component 0 of the next tile
    fft_io<T, N, W, NTH, TileAddr<N, W>, false>(
        A, B, tws, [&](int pos, int col) { return stg[pos * W + col]; }, nl_store(c),
        [&]() {
          if (c < 2 || (LES && a.les)) {
            prefetch(tile, c + 1, stg);
          } else {
            if (tile + (int)gridDim.x < ntiles) prefetch(tile + gridDim.x, 0, stg);
            stage_pass(0);
            stage_pass(1);
          }
        });
  }
  if constexpr (LES) {
    // fused LES stage: x-forward of the six stress components (xx, yy, zz,
    // xy, xz, yz), accumulated into s_i = k_j tau_hat_ij in F[3..5]
    // (the first contribution of each s_i writes, the later ones add)
    if (a.les) {
      const T kyl = a.k.ky[full_pos(j, g.hy, g.My, g.Ny)];
#pragma unroll 1
      for (int c = 3; c < 9; ++c) {
        cp_async_wait_all();
        __syncthreads();
        fft_io<T, N, W, NTH, TileAddr<N, W>, false>(
            A, B, tws, [&](int pos, int col) { return stg[pos * W + col]; },
            [&](int pos, int col, V2<T> v) {
              const int row = compact_row(pos, g.hx, g.Mx, N);
              if (row < 0) return;
              const int z = z0 + col;
              const T kx = a.k.kx[pos], kz = z < g.Mz ? a.k.kz[z] : T(0);
              V2<T>* s0 = F + 3 * MW + row * W + col;
              V2<T>* s1 = s0 + MW;
              V2<T>* s2 = s1 + MW;
              switch (c) {
                case 3: *s0 = cscale(v, kx); break;
                case 4: *s1 = cscale(v, kyl); break;
                case 5: *s2 = cscale(v, kz); break;
                case 6: *s0 = cadd(*s0, cscale(v, kyl)); *s1 = cadd(*s1, cscale(v, kx)); break;
                case 7: *s0 = cadd(*s0, cscale(v, kz)); *s2 = cadd(*s2, cscale(v, kx)); break;
                default: *s1 = cadd(*s1, cscale(v, kz)); *s2 = cadd(*s2, cscale(v, kyl)); break;
              }
            },
            [&]() {
              if (c < 8) prefetch(tile, c + 1, stg);
              else if (tile + (int)gridDim.x < ntiles) prefetch(tile + gridDim.x, 0, stg);
            });
      }
    }
  }
  if constexpr (!REGS) __syncthreads();  // F complete

  const int fy = full_pos(j, g.hy, g.My, g.Ny);
  const T ky = a.k.ky[fy];
  const T cf = (a.forcing == 2 || a.forcing == 3) ? T(a.coef[0]) : T(0);
  double sE = 0.0, sO = 0.0, sB = 0.0;
  const long long cbase = (long long)j * g.Mzp + z0;
  if constexpr (REGS) {
    const int col = threadIdx.x % W, b = threadIdx.x / W;
    const int z = z0 + col;
    const bool zok = z < g.Mz;
    const T kz = zok ? __ldg(a.k.kz + z) : T(0);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      // pass r's copies are done (only pass r+1's may be pending) and every
      // thread has left pass r-1, whose slot now takes pass r+2
      cp_async_wait_group<1>();
      __syncthreads();
      if (r + 2 < 8) stage_pass(r + 2);
      else cp_async_commit();  // empty group: keeps one group per pass
      const V2<T>* slot = F + (r % 3) * p3_ring_slot<N, W>() + b * W + col;
      V2<T> us[3], ac[3], uu[3];
      const int pos = b + r * (N / 8);
      const int i = compact_row(pos, g.hx, g.Mx, N);
      const bool ok = zok && i >= 0;
      const long long o = cbase + (long long)i * a.c_x + col;
      V2<T> du[3] = {f[0][r], f[1][r], f[2][r]};
      V2<T> ns[3] = {czero<T>(), czero<T>(), czero<T>()};
      if (ok) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          us[c] = slot[c * (N / 8) * W];
          if (a.stage >= 2) {
            ac[c] = slot[(3 + c) * (N / 8) * W];
            uu[c] = slot[(6 + c) * (N / 8) * W];
          }
        }
        p3_point(a, pos, fy, z, ky, kz, cf, o, du, us, ac, uu, ns, sE, sO, sB);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) f[c][r] = ns[c];
    }
  } else {
    // two elements per pass: all their state loads are in flight together
    for (int e0 = threadIdx.x; e0 < MW; e0 += 2 * NTH) {
      V2<T> us[2][3], ac[2][3], uu[2][3];
      long long idx[2];
      bool ok[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int e = e0 + h * NTH;
        const int i = e / W, col = e % W;
        ok[h] = e < MW && z0 + col < g.Mz;
        idx[h] = cbase + (long long)i * a.c_x + col;
        if (ok[h]) p3_load(a, idx[h], us[h], ac[h], uu[h]);
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int e = e0 + h * NTH;
        if (e >= MW) continue;
        const int i = e / W, col = e % W;
        V2<T> ns[3] = {czero<T>(), czero<T>(), czero<T>()};
        if (ok[h]) {
          V2<T> du[3] = {F[e], F[MW + e], F[2 * MW + e]};
          if constexpr (LES) {
            if (a.les) {  // f = -i k_j tau_hat_ij: added here, held for the later stages
#pragma unroll
              for (int c = 0; c < 3; ++c) {
                const V2<T> fc = cmul_mi(F[(3 + c) * MW + e]);
                du[c] = cadd(du[c], fc);
                a.fext_out[c * a.c_c + idx[h]] = fc;
              }
            }
          }
          p3_point(a, full_pos(i, g.hx, g.Mx, N), fy, z0 + col, ky, __ldg(a.k.kz + z0 + col), cf, idx[h], du, us[h],
                   ac[h], uu[h], ns, sE, sO, sB);
        }
        if (a.fuse_p1) {
#pragma unroll
          for (int c = 0; c < 3; ++c) F[c * MW + e] = ns[c];
        }
      }
    }
  }
  if (a.partial) {
    block_sum3_f64(sE, sO, sB, red);
    if (threadIdx.x == 0) {
      a.partial[3 * tile + 0] = sE;
      a.partial[3 * tile + 1] = sO;
      a.partial[3 * tile + 2] = sB;
    }
  }
  if constexpr (REGS) {
    if (a.fuse_p1)
      p1_body<T, N, W, NTH>([&](int c, int, int, int r) { return f[c][r]; }, A, B, j, z0, g, a.k, tws, a.t6, a.t6_c,
                            a.t6_x);
  } else {
    __syncthreads();  // F complete; A/B free for the next tile or the fused x-inverse
    if constexpr (LES) {
      if (a.fuse_p1 == 2) {  // the next stage is a fused LES stage
        p1les_body<T, N, W, NTH>(
            [&](int c, int pos, int col, int) {
              const int row = compact_row(pos, g.hx, g.Mx, N);
              return row >= 0 ? F[c * MW + row * W + col] : czero<T>();
            },
            A, B, j, z0, g, a.k, tws, a.t6, a.t6_c, a.t6_x);
        return;
      }
    }
    if (a.fuse_p1)
      p1_body<T, N, W, NTH>(
          [&](int c, int pos, int col, int) {
            const int row = compact_row(pos, g.hx, g.Mx, N);
            return row >= 0 ? F[c * MW + row * W + col] : czero<T>();
          },
          A, B, j, z0, g, a.k, tws, a.t6, a.t6_c, a.t6_x);
  }
}

template <typename T, int N, int W, int NTH>
__global__ void __launch_bounds__(NTH) k_p3(P3Args<T> a, int nzt, int ntiles) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[96];
  V2<T>* A = reinterpret_cast<V2<T>*>(smem_raw);
  V2<T>* B = A + skew8_slots(N, W);
  V2<T>* stg = B + skew8_slots(N, W);  // staged N x W column of the next nl component
  V2<T>* tws = stg + N * W;
  V2<T>* F = tws + (tw_size<false>(N) + 1) / 2 * 2;  // 3 x Mx x W, or the register mode's ring
  fill_stage_twiddles<T, N, false, NTH>(tws, a.tw);
  pdl_wait();
  pdl_trigger();
  if (blockIdx.x < ntiles) {
    const int jj = blockIdx.x / nzt, zz = (blockIdx.x % nzt) * W;
    const V2<T>* src = a.t3 + (long long)jj * a.g.Mzp + zz;
    constexpr int VPC = 16 / sizeof(V2<T>), CPR = W / VPC;
    for (int e = threadIdx.x; e < N * CPR; e += NTH) {
      const int row = e / CPR, ch = e % CPR;
      cp_async16(stg + row * W + ch * VPC, src + (long long)row * a.t_x + ch * VPC);
    }
    cp_async_commit();
  }
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int j = tile / nzt, z0 = (tile % nzt) * W;
    p3_tile<T, N, W, NTH>(a, A, B, tws, F, red, j, z0, tile, stg, nzt, ntiles);
  }
  cp_async_wait_all();
}

// ---------------------------------------------------------------------------
// k_p3m: P3 for float32 columns of 512 points, two 256-thread CTAs per SM,
// with the tile's spectral values parked in tensor memory (TMEM).
//
// The register-mode k_p3 keeps the three nonlinear-term components of a
// thread's positions in registers from the x-forward through the epilogue to
// the fused x-inverse.  That needs one butterfly per thread (512 threads per
// 8-column tile), and with its staging ring one CTA fills an SM, so every
// stage barrier idles the whole SM.  Here a thread owns two butterflies per
// stage (256 threads per tile) and parks what it would hold -- 3 components x
// 16 positions, then the outputs of one inverse transform that the curl needs
// later -- in its own TMEM lane: 128 32-bit columns per thread, 256 per CTA,
// so two CTAs take the SM's 512 columns and one CTA's barriers overlap the
// other's work.  The epilogue's state rows are staged pass by pass into the
// two FFT buffers, which are idle between the forward and inverse transforms.
//
// TMEM columns of a thread (from its base): component c of position
// b_i + r N/8 (butterfly i = 0, 1, b_i = threadIdx.x / W + i * 256 / W) at
// 32 c + 16 i + 2 r (re, im); columns 96 + 16 i + 2 r hold the kept outputs of
// an inverse transform.  Warps w and w + 4 share TMEM lanes 32 (w % 4) .. +31
// and take columns [0, 128) and [128, 256) of the CTA's allocation.
// ---------------------------------------------------------------------------
constexpr int P3M_THREADS = 256;
constexpr int P3M_COLS = 256;  // TMEM columns per CTA

template <int N, int W> __host__ __device__ constexpr bool p3m_fits() {
  return fft_radix(N, 0) == 8 && fft_radix(N, fft_nstages(N) - 1) == 8 && (N / 8) * W == 2 * P3M_THREADS &&
         p3_ring_slot<N, W>() <= skew8_slots(N, W);
}

// x-inverse of the new stage input (in TMEM) and of w = i k x u, as p1_body.
template <int N, int W>
__device__ __forceinline__ void p1m_body(float2* A, float2* B, int j, int z0, const Geom& g, const KTab<float>& kt,
                                         const float2* tws, float2* t6, long long t_c, long long t_x, uint32_t tm) {
  constexpr int NTH = P3M_THREADS;
  const int fy = full_pos(j, g.hy, g.My, g.Ny);
  const float ky = kt.ky[fy];
  float2* out = t6 + (long long)j * g.Mzp + z0;
  const int z = z0 + threadIdx.x % W;  // NTH is a multiple of W: the column of both butterflies
  const float kz = z < g.Nzh ? kt.kz[z] : 0.f;
  auto put = [&](int q, int pos, int col, float2 v) { out[q * t_c + (long long)pos * t_x + col] = v; };
  float lb[16], kb[8], ob[16];
  // first-stage loader of component c (times kx when kxs): the 8 values of
  // butterfly i come from TMEM in one load
  auto src = [&](int c, bool kxs) {
    return [&, c, kxs](int pos, int, int r, int i) {
      if (r == 0) tc::tmem_ld16(tm + 32 * c + 16 * i, lb);
      const float2 v = make_float2(lb[2 * r], lb[2 * r + 1]);
      return kxs ? cscale(v, kt.kx[pos]) : v;
    };
  };
  auto kept = [&](int r, int i) {  // in two halves: fewer live registers in the last stage
    if (r % 4 == 0) tc::tmem_ld8(tm + 96 + 16 * i + 2 * r, kb);
    return make_float2(kb[2 * (r % 4)], kb[2 * (r % 4) + 1]);
  };
  auto keep = [&](float2 v, int r, int i) {
    ob[2 * r] = v.x;
    ob[2 * r + 1] = v.y;
    if (r == 7) tc::tmem_st16(tm + 96 + 16 * i, ob);
  };
  // u_x (kept)
  fft_io<float, N, W, NTH, TileAddr<N, W>, true>(A, B, tws, src(0, false), [&](int pos, int col, float2 v, int r, int i) {
    put(0, pos, col, v);
    keep(v, r, i);
  });
  tc::tmem_wait_st();
  // kx u_y -> w_z = i (X_y - ky u_x)
  fft_io<float, N, W, NTH, TileAddr<N, W>, true>(A, B, tws, src(1, true), [&](int pos, int col, float2 v, int r, int i) {
    put(5, pos, col, cmul_i(csub(v, cscale(kept(r, i), ky))));
  });
  // kx u_z -> w_y = i (kz u_x - X_z)
  fft_io<float, N, W, NTH, TileAddr<N, W>, true>(A, B, tws, src(2, true), [&](int pos, int col, float2 v, int r, int i) {
    put(4, pos, col, cmul_i(csub(cscale(kept(r, i), kz), v)));
  });
  // u_y (kept)
  fft_io<float, N, W, NTH, TileAddr<N, W>, true>(A, B, tws, src(1, false), [&](int pos, int col, float2 v, int r, int i) {
    put(1, pos, col, v);
    keep(v, r, i);
  });
  tc::tmem_wait_st();
  // u_z -> w_x = i (ky u_z - kz u_y)
  fft_io<float, N, W, NTH, TileAddr<N, W>, true>(A, B, tws, src(2, false), [&](int pos, int col, float2 v, int r, int i) {
    put(2, pos, col, v);
    put(3, pos, col, cmul_i(csub(cscale(v, ky), cscale(kept(r, i), kz))));
  });
}

// State-array tensor maps of k_p3m's epilogue ring (see p3m_state_map): the
// stage input (u for stages 0/1, s after), the accumulator and u.
struct P3mMaps {
  CUtensorMap us, acc, u;
};

// One (ky row, z tile) of k_p3m.  stg holds the staged first nl component;
// the ring slots' mbarriers are mb0 and mb0 + 8, and bit k of ph is slot k's
// phase.  False when a ring wait gave up (the CTA then stops).
template <int N, int W>
__device__ __forceinline__ bool p3m_tile(const P3Args<float>& a, float2* A, float2* B, const float2* tws,
                                         double* red, int j, int z0, int tile, float2* stg, int nzt, int ntiles,
                                         uint32_t tm, const P3mMaps& maps, uint32_t mb0, uint32_t& ph) {
  constexpr int NTH = P3M_THREADS, NB = N / 8;
  const Geom& g = a.g;
  constexpr int CPR = W / 2;  // 16-byte chunks per row
  auto prefetch = [&](int t, int c) {
    const int jj = t / nzt, zz = (t % nzt) * W;
    const float2* src = a.t3 + c * a.t_c + (long long)jj * g.Mzp + zz;
    for (int e = threadIdx.x; e < N * CPR; e += NTH) {
      const int row = e / CPR, ch = e % CPR;
      cp_async16(stg + row * W + ch * 2, src + (long long)row * a.t_x + ch * 2);
    }
    cp_async_commit();
  };
  const long long cbase = (long long)j * g.Mzp + z0;
  const int nq = a.stage <= 1 ? 3 : 9;  // (array, component): u | s, acc, u
  // the state rows the epilogue reads, into L2 while the forward transforms run
  for (int q = 0; q < nq; ++q) {
    const float2* arr = q < 3 ? (a.stage <= 1 ? a.u : a.s) : (q < 6 ? a.acc : a.u);
    const float2* base = arr + (q % 3) * a.c_c + cbase;
    for (int i = threadIdx.x; i < g.Mx; i += NTH) prefetch_l2(base + (long long)i * a.c_x, W * sizeof(float2));
  }
  // x-forward of the three nl components; each thread's last-stage outputs go to TMEM
#pragma unroll 1
  for (int c = 0; c < 3; ++c) {
    cp_async_wait_all();
    __syncthreads();
    float ob[16];
    fft_io<float, N, W, NTH, TileAddr<N, W>, false>(
        A, B, tws, [&](int pos, int col) { return stg[pos * W + col]; },
        [&](int, int, float2 v, int r, int i) {
          ob[2 * r] = v.x;
          ob[2 * r + 1] = v.y;
          if (r == 7) tc::tmem_st16(tm + 32 * c + 16 * i, ob);
        },
        [&]() {
          if (c < 2) prefetch(tile, c + 1);
          else if (tile + (int)gridDim.x < ntiles) prefetch(tile + gridDim.x, 0);
        });
  }
  tc::tmem_wait_st();

  // epilogue: pass r covers positions r N/8 .. r N/8 + N/8 - 1 (b_i + r N/8 of
  // every thread); passes whose positions are all outside the stored rows are
  // skipped.  The state rows of a pass are staged into A or B (a 2-slot ring),
  // the next pass's while this one is computed: one thread issues one TMA box
  // per state array (W columns x 1 ky row x N/8 compact rows x 3 components),
  // counted in bytes on the slot's mbarrier.  The box starts at the compact
  // row of the pass's first position in the half it begins in; rows of a box
  // that fall in the 2/3-rule gap or past the array land at positions that are
  // not stored (never read) or are zero-filled by the TMA unit.
  auto stored = [&](int r) {  // does pass r hold a stored row (uniform)
    return r * NB < g.hx || (r + 1) * NB > g.hx + (N - g.Mx);
  };
  auto next_pass = [&](int r) {  // first pass >= r with stored rows (8: none)
    while (r < 8 && !stored(r)) ++r;
    return r;
  };
  const int narr = a.stage <= 1 ? 1 : 3;
  auto stage_pass = [&](int r, int k) {  // pass r into slot k (no-op for r = 8)
    if (r < 8 && threadIdx.x == 0) {
      float2* slot = k ? B : A;
      const int x0 = r * NB < g.hx ? r * NB : r * NB - (N - g.Mx);
      tma::fence_async_smem();  // the slot's earlier generic accesses come first
      const uint32_t mbk = mb0 + 8u * k;
      tma::mbar_expect_tx(mbk, (uint32_t)(narr * 3 * NB * W * sizeof(float2)));
      tma::load4(slot, &maps.us, z0, j, x0, 0, mbk);
      if (narr == 3) {
        tma::load4(slot + 3 * NB * W, &maps.acc, z0, j, x0, 0, mbk);
        tma::load4(slot + 6 * NB * W, &maps.u, z0, j, x0, 0, mbk);
      }
    }
  };
  const int fy = full_pos(j, g.hy, g.My, g.Ny);
  const float ky = a.k.ky[fy];
  const float cf = (a.forcing == 2 || a.forcing == 3) ? (float)a.coef[0] : 0.f;
  double sE = 0.0, sO = 0.0, sB = 0.0;
  const int col = threadIdx.x % W, b0 = threadIdx.x / W;
  const int z = z0 + col;
  const bool zok = z < g.Mz;
  const float kz = zok ? __ldg(a.k.kz + z) : 0.f;
  __syncthreads();  // every thread has left the last forward stage: A and B are free
  int rc = next_pass(0);
  int rn = next_pass(rc + 1);
  stage_pass(rc, 0);
  stage_pass(rn, 1);
  const float zeros[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  int k = 0;
#pragma unroll 1
  for (int r = 0; r < 8; ++r) {
    if (r != rc) {  // no stored rows: the new stage input is zero here
      tc::tmem_st2x3(tm + 2 * r, 32, zeros);
      tc::tmem_st2x3(tm + 16 + 2 * r, 32, zeros);
      continue;
    }
    const int sk = k & 1;
    float2* slot = sk ? B : A;
    {
      // the pass's boxes have landed (a verdict shared by the block)
      const uint32_t mbk = mb0 + 8u * sk, par = (ph >> sk) & 1u;
      const bool ok = __syncthreads_and(tma::mbar_wait(mbk, par, g_axis_wait_limit)) != 0;
      ph ^= 1u << sk;
      if (!ok) {
        if (threadIdx.x == 0) atomicExch(&g_axis_timeout, 1);
        tma::mbar_wait(mbk, par, AXIS_WAIT);  // the copies in flight, once more with a limit
        if (rn < 8) tma::mbar_wait(mb0 + 8u * (sk ^ 1), (ph >> (sk ^ 1)) & 1u, AXIS_WAIT);
        tc::tmem_wait_st();
        return false;
      }
    }
    float d[12];
    tc::tmem_ld2x3x2(tm + 2 * r, 32, 16, d);  // [6 i + 2 c]: component c of butterfly i
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int lb = b0 + i * (NTH / W);
      const int pos = lb + r * NB;
      const int row = compact_row(pos, g.hx, g.Mx, N);
      float2 ns[3] = {czero<float>(), czero<float>(), czero<float>()};
      if (zok && row >= 0) {
        const float2* sl = slot + lb * W + col;
        float2 us[3], ac[3], uu[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          us[c] = sl[c * NB * W];
          if (a.stage >= 2) {
            ac[c] = sl[(3 + c) * NB * W];
            uu[c] = sl[(6 + c) * NB * W];
          }
        }
        float2 du[3] = {make_float2(d[6 * i], d[6 * i + 1]), make_float2(d[6 * i + 2], d[6 * i + 3]),
                        make_float2(d[6 * i + 4], d[6 * i + 5])};
        const long long o = cbase + (long long)row * a.c_x + col;
        p3_point(a, pos, fy, z, ky, kz, cf, o, du, us, ac, uu, ns, sE, sO, sB);
      }
      const float nv[6] = {ns[0].x, ns[0].y, ns[1].x, ns[1].y, ns[2].x, ns[2].y};
      tc::tmem_st2x3(tm + 16 * i + 2 * r, 32, nv);
    }
    __syncthreads();  // the slot is read: it takes the pass after next
    const int r2 = next_pass(rn + 1);
    stage_pass(r2, sk);
    rc = rn;
    rn = r2;
    ++k;
  }
  tc::tmem_wait_st();
  if (a.partial) {
    block_sum3_f64(sE, sO, sB, red);
    if (threadIdx.x == 0) {
      a.partial[3 * tile + 0] = sE;
      a.partial[3 * tile + 1] = sO;
      a.partial[3 * tile + 2] = sB;
    }
  }
  if (a.fuse_p1) p1m_body<N, W>(A, B, j, z0, g, a.k, tws, a.t6, a.t6_c, a.t6_x, tm);
  return true;
}

template <int N, int W>
__global__ void __launch_bounds__(P3M_THREADS, 2) k_p3m(P3Args<float> a, int nzt, int ntiles,
                                                       const __grid_constant__ P3mMaps maps) {
  static_assert(p3m_fits<N, W>(), "two radix-8 butterflies per thread at the first and last stage");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ double red[96];
  __shared__ uint32_t tslot;
  __shared__ __align__(8) uint64_t rbar[2];
  // the ring's TMA boxes land in A and B: 128-byte aligned by hand (the
  // dynamic shared memory follows the static variables with 16-byte alignment
  // only; p3m_smem reserves the 128 bytes)
  float2* A = reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
  float2* B = A + skew8_slots(N, W);
  float2* stg = B + skew8_slots(N, W);  // staged N x W column of the next nl component
  float2* tws = stg + N * W;
  fill_stage_twiddles<float, N, false, P3M_THREADS>(tws, a.tw);
  const int warp = threadIdx.x >> 5;
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(&tslot), P3M_COLS);
  const uint32_t mb0 = tma::smem_u32(&rbar[0]);  // rbar[1] at mb0 + 8
  if (threadIdx.x == 0) {
    tma::mbar_init(mb0, 1);
    tma::mbar_init(mb0 + 8, 1);
  }
  tma::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tm = tslot + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(warp >> 2) * 128;
  uint32_t ph = 0;
  pdl_wait();
  pdl_trigger();
  if (blockIdx.x < ntiles) {
    const int jj = blockIdx.x / nzt, zz = (blockIdx.x % nzt) * W;
    const float2* src = a.t3 + (long long)jj * a.g.Mzp + zz;
    constexpr int CPR = W / 2;
    for (int e = threadIdx.x; e < N * CPR; e += P3M_THREADS) {
      const int row = e / CPR, ch = e % CPR;
      cp_async16(stg + row * W + ch * 2, src + (long long)row * a.t_x + ch * 2);
    }
    cp_async_commit();
  }
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int j = tile / nzt, z0 = (tile % nzt) * W;
    if (!p3m_tile<N, W>(a, A, B, tws, red, j, z0, tile, stg, nzt, ntiles, tm, maps, mb0, ph)) break;
  }
  cp_async_wait_all();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tslot, P3M_COLS);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

template <typename F> cudaError_t dispatch_len(int N, F&& f) {
  switch (N) {
    case 4: return f(std::integral_constant<int, 4>{});
    case 8: return f(std::integral_constant<int, 8>{});
    case 16: return f(std::integral_constant<int, 16>{});
    case 32: return f(std::integral_constant<int, 32>{});
    case 64: return f(std::integral_constant<int, 64>{});
    case 128: return f(std::integral_constant<int, 128>{});
    case 256: return f(std::integral_constant<int, 256>{});
    case 512: return f(std::integral_constant<int, 512>{});
    case 1024: return f(std::integral_constant<int, 1024>{});
    default: return cudaErrorInvalidValue;
  }
}

// P1 shared memory: A, B, the twiddles and the 3 staged components (N x W
// each); P3: A, B, the staged nl column (N x W), the twiddles and, in
// shared-memory mode, the 3 compact tiles (Mx x W).  (Twiddle slots rounded to
// an even count keep what follows 16-byte aligned.)
template <int N> constexpr int tw_slots_even() { return (tw_size<false>(N) + 1) / 2 * 2; }
template <typename T, int N> size_t p1_smem(int W) {
  return sizeof(V2<T>) * ((size_t)2 * skew8_slots(N, W) + 3 * N * W + tw_slots_even<N>());
}
template <typename T, int N, int W, int NTH> size_t p3_smem(int Mx) {
  const size_t f = p3_in_regs<N, W, NTH>() ? (size_t)3 * p3_ring_slot<N, W>()
                                           : (size_t)(p3_les<T, N, W, NTH>() ? 6 : 3) * Mx * W;
  return sizeof(V2<T>) * ((size_t)2 * skew8_slots(N, W) + N * W + tw_slots_even<N>() + f);
}
template <typename T, int N, int W, bool PF> constexpr size_t axis_smem() {
  // + 128 bytes: the staging tile is aligned to 128 bytes
  return sizeof(V2<T>) * (2 * skew8_slots(N, W) + (PF ? N * W : 0) + tw_slots_even<N>()) + (PF ? 128 : 0);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link to
// the driver library).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
    else
      cudaGetLastError();
  }
  return fn;
}

// Tensor map over rows [row0, row0 + rows) of a (c, o, row, z) array of
// complex values: dims (z in 8-byte elements, row, o, c), box (W columns, br
// rows, 1, 1).  False if the layout cannot be described (the caller stages
// with cp.async instead).
template <typename T>
bool axis_map(CUtensorMap* m, const V2<T>* base, long long cols, int rows, int no, int nc, long long s_a,
              long long s_o, long long s_c, int W, int br) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc || rows < 1) return false;
  constexpr int XE = sizeof(V2<T>) / 8;
  const cuuint64_t dims[4] = {(cuuint64_t)(cols * XE), (cuuint64_t)rows, (cuuint64_t)no, (cuuint64_t)nc};
  const cuuint64_t strides[3] = {(cuuint64_t)(s_a * sizeof(V2<T>)), (cuuint64_t)(s_o * sizeof(V2<T>)),
                                 (cuuint64_t)(s_c * sizeof(V2<T>))};
  const cuuint32_t box[4] = {(cuuint32_t)(W * XE), (cuuint32_t)br, 1, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 4, const_cast<V2<T>*>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <typename T>
cudaError_t launch_axis(int N, bool inv, const AxisArgs<T>& a, int nzt, int no, int nc, cudaStream_t st) {
  return dispatch_len(N, [&](auto nn) {
    constexpr int NN = decltype(nn)::value;
    constexpr int W = tile_w<T>(NN);
    const long long ntiles = (long long)nzt * no * nc;
    if ((inv ? a.Mout : a.Min) != NN) return cudaErrorInvalidValue;  // the full side is all N rows
    // staging needs 16-byte aligned rows and whole tiles inside the source rows
    // (which may extend past the nz valid columns: padded rows)
    const bool pf = (sizeof(V2<T>) == 16 || ((a.s_a | a.s_o | a.s_c) % 2 == 0 &&
                                              ((uintptr_t)a.src % 16) == 0)) &&
                    (long long)nzt * W <= (a.src_cols > 0 ? a.src_cols : a.nz);
    static PerDevice c[6];
    CUtensorMap mA{}, mB{};
    if (pf) {
      // TMA staging when the layout has a tensor map: box rows br (a power of
      // two <= 64) such that the boxes of the two halves do not overlap
      AxisArgs<T> t = a;
      t.pb = a.Min - a.hin;
      t.br = 64;
      auto nb = [](int rows, int br) { return (rows + br - 1) / br; };
      while (t.br > 2 && t.br * (nb(a.hin, t.br) + nb(t.pb, t.br)) > NN) t.br /= 2;
      t.ka = nb(a.hin, t.br);
      t.kb = nb(t.pb, t.br);
      const long long cols = a.src_cols > 0 ? a.src_cols : a.nz;
      const bool tma = a.hin >= 1 && t.pb >= 1 && t.br * (t.ka + t.kb) <= NN && ((uintptr_t)a.src % 16) == 0 &&
                       axis_map<T>(&mA, a.src, cols, a.hin, no, nc, a.s_a, a.s_o, a.s_c, W, t.br) &&
                       axis_map<T>(&mB, a.src + (long long)a.hin * a.s_a, cols, t.pb, no, nc, a.s_a, a.s_o, a.s_c, W,
                                   t.br);
      const size_t smem = axis_smem<T, NN, W, true>();
      if (tma) {
        if (inv)
          return launch_pdl(k_axis<T, NN, W, true, 2>, resident_grid(k_axis<T, NN, W, true, 2>, NT, smem, ntiles, c[4]),
                            NT, smem, st, t, nzt, no, (int)ntiles, mA, mB);
        return launch_pdl(k_axis<T, NN, W, false, 2>, resident_grid(k_axis<T, NN, W, false, 2>, NT, smem, ntiles, c[5]),
                          NT, smem, st, t, nzt, no, (int)ntiles, mA, mB);
      }
      if (inv)
        return launch_pdl(k_axis<T, NN, W, true, 1>, resident_grid(k_axis<T, NN, W, true, 1>, NT, smem, ntiles, c[0]),
                          NT, smem, st, a, nzt, no, (int)ntiles, mA, mB);
      return launch_pdl(k_axis<T, NN, W, false, 1>, resident_grid(k_axis<T, NN, W, false, 1>, NT, smem, ntiles, c[1]),
                        NT, smem, st, a, nzt, no, (int)ntiles, mA, mB);
    } else {
      const size_t smem = axis_smem<T, NN, W, false>();
      if (inv)
        k_axis<T, NN, W, true, 0><<<resident_grid(k_axis<T, NN, W, true, 0>, NT, smem, ntiles, c[2]), NT, smem, st>>>(
            a, nzt, no, (int)ntiles, mA, mB);
      else
        k_axis<T, NN, W, false, 0><<<resident_grid(k_axis<T, NN, W, false, 0>, NT, smem, ntiles, c[3]), NT, smem,
                                     st>>>(a, nzt, no, (int)ntiles, mA, mB);
    }
    return cudaGetLastError();
  });
}

// Polls of the tile-box wait of k_axis on the current device (polls < 0: the
// default).
cudaError_t set_axis_wait_limit(int polls) {
  const int v = polls < 0 ? AXIS_WAIT : polls;
  return cudaMemcpyToSymbol(g_axis_wait_limit, &v, sizeof(int));
}

// Read and clear the flag a TMA wait of k_axis sets when it gives up.
cudaError_t take_axis_timeout(int* flag) {
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_axis_timeout, sizeof(int));
  if (e != cudaSuccess) return e;
  *flag = v;
  const int zero = 0;
  return v ? cudaMemcpyToSymbol(g_axis_timeout, &zero, sizeof(int)) : cudaSuccess;
}

template <typename T> int p3_tile_w(int Nx) {
  int w = 0;
  dispatch_len(Nx, [&](auto nn) { w = tile_wp<T>(decltype(nn)::value); return cudaSuccess; });
  return w;
}

template <typename T> int axis_tile_w(int N) {
  int w = 0;
  dispatch_len(N, [&](auto nn) { w = tile_w<T>(decltype(nn)::value); return cudaSuccess; });
  return w;
}

int p3_num_blocks(const Geom& g, int W) { return (g.Mzp / W) * g.My; }

template <typename K> cudaError_t max_smem(K kernel, int bytes) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
}

template <typename T, int NN, int W, int NTH> cudaError_t launch_p1_v(const P1Args<T>& a, cudaStream_t st) {
  static PerDevice cache, ready;
  cudaError_t e = once_per_device(ready, [] { return max_smem(k_p1<T, NN, W, NTH>, (int)p1_smem<T, NN>(W)); });
  if (e != cudaSuccess) return e;
  const int nzt = a.g.Mzp / W, ntiles = nzt * a.g.My;
  const size_t smem = p1_smem<T, NN>(W);
  return launch_pdl(k_p1<T, NN, W, NTH>, resident_grid(k_p1<T, NN, W, NTH>, NTH, smem, ntiles, cache), NTH, smem, st, a,
                    nzt, ntiles);
}

template <typename T, int NN, int W, int NTH> cudaError_t launch_p3_v(const P3Args<T>& a, cudaStream_t st) {
  static PerDevice cache, ready;
  cudaError_t e =
      once_per_device(ready, [] { return max_smem(k_p3<T, NN, W, NTH>, (int)p3_smem<T, NN, W, NTH>(NN)); });
  if (e != cudaSuccess) return e;
  const int nzt = a.g.Mzp / W, ntiles = nzt * a.g.My;
  const size_t smem = p3_smem<T, NN, W, NTH>(a.g.Mx);
  return launch_pdl(k_p3<T, NN, W, NTH>, resident_grid(k_p3<T, NN, W, NTH>, NTH, p3_smem<T, NN, W, NTH>(NN), ntiles, cache),
                    NTH, smem, st, a, nzt, ntiles);
}

// k_p3m shared memory: A, B, the staged nl column (N x W) and the twiddles,
// plus 128 bytes for aligning A.
template <int N, int W> constexpr size_t p3m_smem() {
  return sizeof(float2) * ((size_t)2 * skew8_slots(N, W) + N * W + tw_slots_even<N>()) + 128;
}

// Tensor map of k_p3m's epilogue ring over a compact state array (3, Mx, My,
// Mzp) of complex values: dims (z, ky row, compact x row, component) in
// 8-byte elements, box (W, 1, rows, 3); the boxes start at multiples of W in
// z (64-byte aligned), the other coordinates may run past the array (zero
// fill).
bool p3m_state_map(CUtensorMap* m, const float2* base, const Geom& g, long long c_x, long long c_c, int W, int rows) {
  EncodeTiledFn enc = encode_tiled();
  if (!enc || ((uintptr_t)base % 16) || g.Mzp % 2) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)g.Mzp, (cuuint64_t)g.My, (cuuint64_t)g.Mx, 3};
  const cuuint64_t strides[3] = {(cuuint64_t)g.Mzp * sizeof(float2), (cuuint64_t)c_x * sizeof(float2),
                                 (cuuint64_t)c_c * sizeof(float2)};
  const cuuint32_t box[4] = {(cuuint32_t)W, 1, (cuuint32_t)rows, 3};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 4, const_cast<float2*>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int NN, int W> cudaError_t launch_p3m_v(const P3Args<float>& a, cudaStream_t st) {
  static PerDevice cache, ready;
  cudaError_t e = once_per_device(ready, [] { return max_smem(k_p3m<NN, W>, (int)p3m_smem<NN, W>()); });
  if (e != cudaSuccess) return e;
  const int nzt = a.g.Mzp / W, ntiles = nzt * a.g.My;
  P3mMaps maps{};
  constexpr int NB = NN / 8;
  if (!p3m_state_map(&maps.us, a.stage <= 1 ? a.u : a.s, a.g, a.c_x, a.c_c, W, NB) ||
      !p3m_state_map(&maps.acc, a.acc, a.g, a.c_x, a.c_c, W, NB) ||
      !p3m_state_map(&maps.u, a.u, a.g, a.c_x, a.c_c, W, NB))
    return cudaErrorInvalidValue;
  // Resident CTAs: the occupancy query counts one CTA per SM for kernels that
  // allocate tensor memory, so the wave is sized from the SM's shared memory
  // and registers, at most 2 per SM (two 256-column TMEM allocations fill it).
  std::atomic<int>* slot = cache.here();
  int wave = slot ? slot->load(std::memory_order_relaxed) : 0;
  if (wave == 0) {
    int dev = 0, sms = 0, smem_sm = 0, regs_sm = 0;
    cudaFuncAttributes fa{};
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess)
      return e;
    if ((e = cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev)) != cudaSuccess) return e;
    if ((e = cudaFuncGetAttributes(&fa, k_p3m<NN, W>)) != cudaSuccess) return e;
    const int by_smem = smem_sm / (int)(p3m_smem<NN, W>() + fa.sharedSizeBytes + 1024);
    const int by_regs = regs_sm / (P3M_THREADS * ((std::max(fa.numRegs, 1) + 7) / 8 * 8));
    wave = std::max(1, std::min(std::min(by_smem, by_regs), 512 / P3M_COLS)) * std::max(sms, 1);
    if (slot) slot->store(wave, std::memory_order_relaxed);
  }
  return launch_pdl(k_p3m<NN, W>, ntiles < wave ? std::max(ntiles, 1) : wave, P3M_THREADS, p3m_smem<NN, W>(), st, a,
                    nzt, ntiles, maps);
}

// Threads per k_p1/k_p3 CTA: 512 (one CTA per SM at 512- and 1024-point
// columns); 256 for columns of at most 128 points, whose tiles have at most
// 128 butterflies per stage, so that the CTA leaves half an SM's registers to
// other work (on small grids, e.g. a closure on a second stream).
template <int N> constexpr int p_threads() { return N <= 128 ? NTP / 2 : NTP; }

template <typename T> cudaError_t launch_p1(const P1Args<T>& a, cudaStream_t st) {
  return dispatch_len(a.g.Nx, [&](auto nn) {
    constexpr int NN = decltype(nn)::value;
    return launch_p1_v<T, NN, tile_wp<T>(NN), p_threads<NN>()>(a, st);
  });
}

template <typename T> cudaError_t launch_p3(const P3Args<T>& a, cudaStream_t st) {
  return dispatch_len(a.g.Nx, [&](auto nn) {
    constexpr int NN = decltype(nn)::value;
    if constexpr (std::is_same<T, float>::value && NN == 512) {
      return launch_p3m_v<NN, tile_wp<float>(NN)>(a, st);
    } else {
      return launch_p3_v<T, NN, tile_wp<T>(NN), p_threads<NN>()>(a, st);
    }
  });
}

template <typename T> cudaError_t prepare_axis_kernels(int Nx) {
  return dispatch_len(Nx, [&](auto nn) {
    constexpr int NN = decltype(nn)::value;
    cudaError_t e;
    constexpr int W = tile_w<T>(NN);
    if ((e = max_smem(k_axis<T, NN, W, true, 2>, (int)axis_smem<T, NN, W, true>())) != cudaSuccess) return e;
    if ((e = max_smem(k_axis<T, NN, W, false, 2>, (int)axis_smem<T, NN, W, true>())) != cudaSuccess) return e;
    if ((e = max_smem(k_axis<T, NN, W, true, 1>, (int)axis_smem<T, NN, W, true>())) != cudaSuccess) return e;
    if ((e = max_smem(k_axis<T, NN, W, false, 1>, (int)axis_smem<T, NN, W, true>())) != cudaSuccess) return e;
    if ((e = max_smem(k_axis<T, NN, W, true, 0>, (int)axis_smem<T, NN, W, false>())) != cudaSuccess) return e;
    return max_smem(k_axis<T, NN, W, false, 0>, (int)axis_smem<T, NN, W, false>());
  });
}

template cudaError_t launch_axis<float>(int, bool, const AxisArgs<float>&, int, int, int, cudaStream_t);
template cudaError_t launch_axis<double>(int, bool, const AxisArgs<double>&, int, int, int, cudaStream_t);
template cudaError_t launch_p1<float>(const P1Args<float>&, cudaStream_t);
template cudaError_t launch_p1<double>(const P1Args<double>&, cudaStream_t);
template cudaError_t launch_p3<float>(const P3Args<float>&, cudaStream_t);
template cudaError_t launch_p3<double>(const P3Args<double>&, cudaStream_t);
template cudaError_t prepare_axis_kernels<float>(int);
template cudaError_t prepare_axis_kernels<double>(int);
template int p3_tile_w<float>(int);
template int p3_tile_w<double>(int);
template int axis_tile_w<float>(int);
template int axis_tile_w<double>(int);

}  // namespace hit
