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
// k_zcross fuses the middle of the RHS (src/hit3d/navierstokes.py:78-89): for RB
// (x, y) rows, the c2r of u and w (6 rows each) runs as one batch whose last
// stage leaves the physical values in shared memory; the forward transform's
// first stage forms u x w from them; its last stage leaves the spectrum in
// shared memory for the r2c post-processing, which writes the three products
// over the first three input components of the same rows.
#include <algorithm>
#include <atomic>
#include <type_traits>

#include "fft_core.cuh"
#include "kernels.h"
#include "mlp_core.cuh"
#include "tma.cuh"
#include "zwarp.cuh"

namespace hit {

template <int H> __host__ __device__ constexpr int z_rows_per_block() {
  return (512 / H) > 32 ? 32 : (512 / H < 1 ? 1 : 512 / H);
}
// threads per block: one per last-stage butterfly of the 3*RB forward rows
template <int H> __host__ __device__ constexpr int z_threads() {
  return ((3 * z_rows_per_block<H>() * (H / fft16_radix(H, fft16_nstages(H) - 1)) + 31) / 32 * 32) < 96
             ? 96
             : ((3 * z_rows_per_block<H>() * (H / fft16_radix(H, fft16_nstages(H) - 1)) + 31) / 32 * 32);
}
// rows of Mzp entries are at most this long (Mzp <= round_up(H+1, 8))
template <int H> __host__ __device__ constexpr int z_row_cap() { return (H + 1 + 7) / 8 * 8; }

// conj-paired pre-processing of one c2r row element k in [0, H).
template <typename T>
__device__ __forceinline__ V2<T> c2r_pre(const V2<T>* row, int k, int H, int Mz, const V2<T>* twz) {
  V2<T> X = k < Mz ? row[k] : czero<T>();
  const int kk = H - k;  // in [1, H]
  V2<T> Y = kk < Mz ? row[kk] : czero<T>();
  if (k == 0) {
    X.y = T(0);
    Y.y = T(0);  // kk == H: Nyquist
  }
  Y.y = -Y.y;  // conj X[H-k]
  const V2<T> s = cadd(X, Y), d = csub(X, Y);
  V2<T> w = twz[k];
  w.y = -w.y;  // e^{+2 pi i k / Nz}
  return cadd(s, cmul_i(cmul(w, d)));
}

// r2c post-processing: output bin k in [0, H] from Z (length H), Z[i] = z(i).
// HALVE = false returns twice the bin (for callers that fold the 1/2 into
// their input scale).
template <typename T, bool HALVE = true, class ZF>
__device__ __forceinline__ V2<T> r2c_post(ZF&& z, int k, int H, const V2<T>* twz) {
  const V2<T> a = z(k == H ? 0 : k);
  V2<T> b = z(k == 0 ? 0 : H - k);
  b.y = -b.y;
  V2<T> E = cadd(a, b), O = cmul_mi(csub(a, b));
  if constexpr (HALVE) {
    E = cscale(E, T(0.5));
    O = cscale(O, T(0.5));
  }
  const V2<T> w = twz[k];  // e^{-2 pi i k / Nz}
  return cadd(E, cmul(w, O));
}

// Shared twiddles of the z kernels: the FFT stage tables (length H, radix-16
// plan) followed by exp(-2 pi i k / Nz) for k in [0, H].
template <int H> __host__ __device__ constexpr int z_tw_slots() { return (tw_size<true>(H) + H + 1 + 1) / 2 * 2; }
// (an even slot count keeps whatever follows the tables 16-byte aligned)
template <typename T, int H, int NTH>
__device__ __forceinline__ void fill_z_twiddles(V2<T>* tws, const V2<T>* __restrict__ tw) {
  fill_stage_twiddles<T, H, true, NTH>(tws, tw);
  V2<T>* twz = tws + tw_size<true>(H);
  for (int k = threadIdx.x; k <= H; k += NTH) twz[k] = tw[k * (TWN / (2 * H))];
  __syncthreads();
}

constexpr int Z_WAIT = 1 << 22;  // mbarrier polls before a TMA wait gives up
__device__ int g_z_timeout = 0;   // set when a TMA wait gave up (hit_device_status)
// Polls of the wait for a row group (hit_set_wait_limit lowers it so that a
// test can make the wait give up); the wait for the copies still in flight
// after a give-up always polls Z_WAIT times.
__device__ int g_z_wait_limit = Z_WAIT;

template <typename T, int H, int RB, int NTZ, int MINB>
__global__ void __launch_bounds__(NTZ, MINB) k_zcross(ZCrossArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  using AD = SkewAddr<skew_ld(H)>;
  V2<T>* buf = reinterpret_cast<V2<T>*>(smem_raw);  // 6*RB columns of AD::LD slots
  V2<T>* tws = buf + 6 * RB * AD::LD;
  const V2<T>* twz = tws + tw_size<true>(H);
  // next group's input rows [q*RB + lr][RS]: entries past Mzp stay zero, so the
  // c2r pre-processing reads X[k] and X[H-k] without checks.  Entries Mz..Mzp-1
  // are the rows' padding columns, which every compact spectral buffer keeps
  // zero (the gather writes zeros there and no RHS kernel writes anything else).
  constexpr int RS = z_row_cap<H>();
  V2<T>* raw = tws + z_tw_slots<H>();
  fill_z_twiddles<T, H, NTZ>(tws, a.tw);
  const int ngroups = (a.nrows + RB - 1) / RB;
  const int Mzp = a.Mzp;
  constexpr int VPC = 16 / sizeof(V2<T>);  // complex values per 16-byte copy
  for (int e = threadIdx.x; e < 6 * RB * RS; e += NTZ)
    if (e % RS >= Mzp) raw[e] = czero<T>();
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  constexpr int NWARP = NTZ / 32;

  // stage the 6 component rows of a group with one bulk TMA copy per row
  // (Mzp entries, a multiple of 8: whole 16-byte chunks), issued by one thread
  // and counted on an mbarrier.  Rows past the end are not loaded: their
  // columns keep stale values, which stay in those columns of the transforms
  // and are never written out.
  __shared__ __align__(8) uint64_t zbar;
  const uint32_t mb = tma::smem_u32(&zbar);
  if (threadIdx.x == 0) tma::mbar_init(mb, 1);
  tma::fence_async_smem();
  __syncthreads();
  auto prefetch = [&](int grp) {
    if (threadIdx.x < 32) {  // warp 0: lane 0 sets the transaction count, the lanes issue the rows
      const long long r0 = (long long)grp * RB;
      const int nin = (int)(a.nrows - r0 < RB ? a.nrows - r0 : RB);
      const uint32_t bytes = (uint32_t)(Mzp * sizeof(V2<T>));
      if (threadIdx.x == 0) tma::mbar_expect_tx(mb, 6u * nin * bytes);
      __syncwarp();
      for (int col = threadIdx.x; col < 6 * RB; col += 32) {
        const int q = col / RB, lr = col % RB;
        if (lr < nin) tma::load_bytes(raw + col * RS, a.buf + q * a.c_stride + (r0 + lr) * Mzp, bytes, mb);
      }
    }
  };

  const int wait_limit = g_z_wait_limit;
  pdl_wait();
  pdl_trigger();
  int grp = blockIdx.x;
  if (grp < ngroups) prefetch(grp);
  uint32_t phase = 0;
  for (; grp < ngroups; grp += gridDim.x) {
    const long long row0 = (long long)grp * RB;
    const bool full = row0 + RB <= a.nrows;
    {
      // the group's rows have landed (a verdict shared by the block)
      const bool ok = __syncthreads_and(tma::mbar_wait(mb, phase, wait_limit)) != 0;
      phase ^= 1;
      if (!ok) {
        if (threadIdx.x == 0) atomicExch(&g_z_timeout, 1);
        tma::mbar_wait(mb, phase ^ 1, Z_WAIT);  // the copies in flight, once more with a limit
        return;
      }
    }

    // c2r of the 6 components of RB rows (column = q*RB + lr) from the staged
    // rows; as soon as every thread holds its first-stage inputs the staging
    // buffer is refilled with the next group while this one is transformed
    const int nxt = grp + gridDim.x;
    fft_ip<T, H, 6 * RB, NTZ, AD, true>(
        buf, tws,
        [&](int k, int col) {
          const V2<T>* row = raw + col * RS;
          V2<T> X = row[k];
          V2<T> Y = row[H - k];
          if (k == 0) {
            X.y = T(0);
            Y.y = T(0);
          }
          Y.y = -Y.y;
          const V2<T> sm = cadd(X, Y), df = csub(X, Y);
          V2<T> w = twz[k];
          w.y = -w.y;
          return cadd(sm, cmul_i(cmul(w, df)));
        },
        [&](int m, int col, V2<T> v) { buf[AD::at(m, col)] = v; },
        [&]() {
          if (nxt < ngroups) prefetch(nxt);
        });

    // r2c of u x w (navierstokes.py:82-86), formed while loading the first
    // stage; the post-processing's 1/2 is folded into the product's scale
    const T s2 = T(0.5) * a.scale * a.scale;
    fft_ip<T, H, 3 * RB, NTZ, AD, false>(
        buf, tws,
        [&](int m, int col) {
          const int c = col / RB, lr = col % RB;
          const int c1 = c == 2 ? 0 : c + 1, c2 = c == 0 ? 2 : c - 1;  // (1,2), (2,0), (0,1)
          const V2<T> ua = buf[AD::at(m, c1 * RB + lr)], ub = buf[AD::at(m, c2 * RB + lr)];
          const V2<T> wa = buf[AD::at(m, (3 + c1) * RB + lr)], wb = buf[AD::at(m, (3 + c2) * RB + lr)];
          V2<T> n;
          n.x = (ua.x * wb.x - ub.x * wa.x) * s2;
          n.y = (ua.y * wb.y - ub.y * wa.y) * s2;
          return n;
        },
        [&](int k, int col, V2<T> v) { buf[AD::at(k, col)] = v; });

    const int Mz = a.Mz;
    for (int col = warp; col < 3 * RB; col += NWARP) {
      const int q = col / RB, lr = col % RB;
      if (full || row0 + lr < a.nrows) {
        V2<T>* out = a.buf + q * a.c_stride + (row0 + lr) * Mzp;
        for (int k = lane; k < Mzp; k += 32)
          out[k] = k < Mz ? r2c_post<T, false>([&](int i) { return buf[AD::at(i, col)]; }, k, H, twz) : czero<T>();
      }
    }
    __syncthreads();  // buf is rewritten by the next group
  }
  cp_async_wait_all();
}

// k_zles: the z pass of the fused LES stage (float32, Nz = 2H in {32, 64,
// 128}).  A CTA of 128 threads takes RB = 128 / Nz (x, y) rows at a time:
//   * c2r of u and the nine velocity gradients g_ij = d_j u_i (12 rows each,
//     staged by bulk TMA copies as in k_zcross);
//   * thread t then owns physical point t of the group (row t / Nz, z = t % Nz):
//     w = (g_21 - g_12, g_02 - g_20, g_10 - g_01), u x w
//     (src/hit3d/navierstokes.py:73-86), and the closure MLP on the tensor cores
//     (mlp::infer_tile: the nine gradients in physical units in, the six SGS
//     stresses out; thread t is TMEM lane t of the 128-point tile);
//   * r2c of the three products and the six stresses, written over the first
//     nine input rows of each (x, y) row.
// The unnormalised inverse transforms leave every physical value times
// Nx Ny Nz: the gradients are scaled back for the MLP, and the products take
// (1/(Nx Ny Nz))^2 / 2, the stresses 1/2 (the r2c post-processing's halving).
constexpr int ZLES_MMA_WAIT = 1 << 22;  // mbarrier polls before an MMA wait gives up

template <int H>
__global__ void __launch_bounds__(128, 4) k_zles(ZLesArgs a) {
  constexpr int NZ = 2 * H, RB = 128 / NZ, NTZ = 128;
  using AD = SkewAddr<skew_ld(H)>;
  constexpr int RS = z_row_cap<H>();
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  mlp::InferSmem& M = *reinterpret_cast<mlp::InferSmem*>(smem_raw);
  float2* buf = reinterpret_cast<float2*>(smem_raw + (sizeof(mlp::InferSmem) + 127) / 128 * 128);
  float2* tws = buf + 12 * RB * AD::LD;
  const float2* twz = tws + tw_size<true>(H);
  float2* raw = tws + z_tw_slots<H>();  // 12 RB staged rows of RS entries
  __shared__ __align__(8) uint64_t zbar;
  const int Mzp = a.Mzp, Mz = a.Mz;
  for (int e = threadIdx.x; e < 12 * RB * RS; e += NTZ)
    if (e % RS >= Mzp) raw[e] = make_float2(0.f, 0.f);
  mlp::infer_setup(M, a.w1t, a.w2t, a.w3t, a.w4t, a.b2, a.b3, a.b4);
  const uint32_t mb = tma::smem_u32(&zbar);
  if (threadIdx.x == 0) tma::mbar_init(mb, 1);
  tma::fence_async_smem();
  fill_z_twiddles<float, H, NTZ>(tws, a.tw);  // ends with __syncthreads
  tc::fence_after_sync();
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  const int ngroups = (a.nrows + RB - 1) / RB;
  auto prefetch = [&](int grp) {
    if (threadIdx.x < 32) {
      const long long r0 = (long long)grp * RB;
      const int nin = (int)(a.nrows - r0 < RB ? a.nrows - r0 : RB);
      const uint32_t bytes = (uint32_t)(Mzp * sizeof(float2));
      if (threadIdx.x == 0) tma::mbar_expect_tx(mb, 12u * nin * bytes);
      __syncwarp();
      for (int col = threadIdx.x; col < 12 * RB; col += 32) {
        const int q = col / RB, lr = col % RB;
        if (lr < nin) tma::load_bytes(raw + col * RS, a.buf + q * a.c_stride + (r0 + lr) * Mzp, bytes, mb);
      }
    }
  };
  const int wait_limit = g_z_wait_limit;
  pdl_wait();
  pdl_trigger();
  int grp = blockIdx.x;
  if (grp < ngroups) prefetch(grp);
  uint32_t phase = 0, mphase = 0;
  bool ok = true;
  for (; grp < ngroups && ok; grp += gridDim.x) {
    const long long row0 = (long long)grp * RB;
    {
      const bool landed = __syncthreads_and(tma::mbar_wait(mb, phase, wait_limit)) != 0;
      phase ^= 1;
      if (!landed) {
        if (threadIdx.x == 0) atomicExch(&g_z_timeout, 1);
        tma::mbar_wait(mb, phase ^ 1, Z_WAIT);  // the copies in flight, once more with a limit
        break;
      }
    }
    const int nxt = grp + gridDim.x;
    fft_ip<float, H, 12 * RB, NTZ, AD, true>(
        buf, tws,
        [&](int k, int col) {
          const float2* row = raw + col * RS;
          float2 X = row[k];
          float2 Y = row[H - k];
          if (k == 0) {
            X.y = 0.f;
            Y.y = 0.f;
          }
          Y.y = -Y.y;
          const float2 sm = cadd(X, Y), df = csub(X, Y);
          float2 w = twz[k];
          w.y = -w.y;
          return cadd(sm, cmul_i(cmul(w, df)));
        },
        [&](int m, int col, float2 v) { buf[AD::at(m, col)] = v; },
        [&]() {
          if (nxt < ngroups) prefetch(nxt);
        });
    // this thread's physical point
    const int lr = threadIdx.x / NZ, zp = threadIdx.x % NZ, m = zp >> 1, hf = zp & 1;
    const float* bf = reinterpret_cast<const float*>(buf);
    auto val = [&](int q) { return bf[2 * AD::at(m, q * RB + lr) + hf]; };
    float u[3], gr[9], gp[9];
#pragma unroll
    for (int q = 0; q < 3; ++q) u[q] = val(q);
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      gr[q] = val(3 + q);
      gp[q] = gr[q] * a.scale;
    }
    const float w[3] = {gr[7] - gr[5], gr[2] - gr[6], gr[3] - gr[1]};
    const float s2 = 0.5f * a.scale * a.scale;
    float nl[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int c1 = c == 2 ? 0 : c + 1, c2 = c == 0 ? 2 : c - 1;  // (1,2), (2,0), (0,1)
      nl[c] = (u[c1] * w[c2] - u[c2] * w[c1]) * s2;
    }
    float tau[6];
    mlp::infer_tile(M, gp, tau, mphase, ok, ZLES_MMA_WAIT);  // all threads; its first MMA syncs the block
    float* bw = reinterpret_cast<float*>(buf);
#pragma unroll
    for (int c = 0; c < 3; ++c) bw[2 * AD::at(m, c * RB + lr) + hf] = nl[c];
#pragma unroll
    for (int c = 0; c < 6; ++c) bw[2 * AD::at(m, (3 + c) * RB + lr) + hf] = 0.5f * tau[c];
    __syncthreads();
    fft_ip<float, H, 9 * RB, NTZ, AD, false>(
        buf, tws, [&](int mm, int col) { return buf[AD::at(mm, col)]; },
        [&](int k, int col, float2 v) { buf[AD::at(k, col)] = v; });
    for (int col = warp; col < 9 * RB; col += NTZ / 32) {
      const int q = col / RB, rr = col % RB;
      if (row0 + rr < a.nrows) {
        float2* out = a.buf + q * a.c_stride + (row0 + rr) * Mzp;
        for (int k = lane; k < Mzp; k += 32)
          out[k] = k < Mz ? r2c_post<float, false>([&](int i) { return buf[AD::at(i, col)]; }, k, H, twz)
                          : make_float2(0.f, 0.f);
      }
    }
    __syncthreads();  // buf is rewritten by the next group
  }
  if (!ok && threadIdx.x == 0) atomicExch(a.err, 1);
  mlp::infer_teardown(M);
}

// k_zwarp: the fused z pass of k_zcross (same inputs, outputs and arithmetic
// per value) with warp-resident transforms (zwarp.cuh), float32, H in {32, 64,
// 128, 256}.  Persistent CTAs of NWARP independent warps; warp g walks the row
// groups g, g + (all warps), ...  A warp stages its group's 6 x ROWS input rows
// (Mzp entries each) with bulk TMA copies issued by its lanes and counted on
// its own mbarrier, and prefetches the next group as soon as the last input
// field has passed through its first transform.  Per lane and row: the six
// c2r transforms (pre-processing from the staged rows), u x w in registers as
// the fields arrive (u first, then each w adds its terms), three r2c
// transforms and the post-processing with the conjugate partner fetched by a
// shuffle; outputs are written over the first three input fields of the row.

constexpr int ZW_MINB = 3;  // CTAs per SM the register budget is sized for
// DA: the dealiased layout, Mz = Nz/3 + 1 and Mzp = Mz rounded up to 8 as
// compile-time constants, so the bounds of the pre-processing loads and of
// the outputs fold into each value's position range (known-zero inputs are
// not loaded, outputs past the row are not formed).
template <int H> constexpr int zw_da_mz() { return (2 * H) / 3 + 1; }
template <int H, int NWARP, bool DA>
__global__ void __launch_bounds__(NWARP * 32, ZW_MINB) k_zwarp(ZCrossArgs<float> a) {
  using Z = ZW<H>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bars[NWARP];
  float2* tws = reinterpret_cast<float2*>(smem_raw);
  const int Mz = DA ? zw_da_mz<H>() : a.Mz;
  const int Mzp = DA ? (zw_da_mz<H>() + 7) / 8 * 8 : a.Mzp;
  // k < bound for a k known to lie in [lo, hi] (lo, hi compile-time)
  auto below = [](int k, int lo, int hi, int bound) { return hi < bound ? true : (lo >= bound ? false : k < bound); };
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = lane / Z::LPR, b = lane % Z::LPR;
  const ZwMid<H> mid(b);
  float2 wl[7];  // filled once the twiddle tables are in shared memory
  const int stg_slots = 6 * Z::ROWS * Mzp;
  float2* stg = tws + Z::TWS + warp * (stg_slots + Z::ROWS * Z::XS);  // [field][row][Mzp]
  float2* xch = stg + stg_slots + q * Z::XS;
  const float2* twz = tws + Z::TWZ;
  zw_fill_twiddles<H, NWARP * 32>(tws, a.tw);
  const uint32_t mb = tma::smem_u32(&bars[warp]);
  if (lane == 0) tma::mbar_init(mb, 1);
  tma::fence_async_smem();
  __syncthreads();
  zw_last_twiddles<H>(wl, tws, b);

  const int wait_limit = g_z_wait_limit;
  const long long ngroups = a.nrows / Z::ROWS;
  const long long nwarps = (long long)gridDim.x * NWARP;
  const uint32_t row_bytes = (uint32_t)(Mzp * sizeof(float2));
  auto prefetch = [&](long long grp) {
    if (lane == 0) tma::mbar_expect_tx(mb, 6u * Z::ROWS * row_bytes);
    __syncwarp();
    for (int i = lane; i < 6 * Z::ROWS; i += 32) {  // i = field * ROWS + row (48 rows at H = 32)
      const int c = i / Z::ROWS, rr = i % Z::ROWS;
      tma::load_bytes(stg + i * Mzp, a.buf + c * a.c_stride + (grp * Z::ROWS + rr) * Mzp, row_bytes, mb);
    }
  };

  pdl_wait();
  pdl_trigger();
  long long grp = (long long)blockIdx.x * NWARP + warp;
  if (grp < ngroups) prefetch(grp);
  uint32_t phase = 0;
  const float s2 = 0.5f * a.scale * a.scale;  // both inverse normalisations and the r2c 1/2
  for (; grp < ngroups; grp += nwarps) {
    {
      const bool ok = __all_sync(0xffffffffu, tma::mbar_wait(mb, phase, wait_limit));
      phase ^= 1;
      if (!ok) {
        if (lane == 0) atomicExch(&g_z_timeout, 1);
        tma::mbar_wait(mb, phase ^ 1, Z_WAIT);  // the copies in flight, once more with a limit
        return;
      }
    }
    float2 u0[8], u1[8], u2[8], n0[8], n1[8], n2[8];
    // e^{-2 pi i k / Nz} of this lane's positions k = b + (H/8) r (zw_wz(wz0,
    // r)) for the pre-processing of the six fields and the post-processing of
    // the three products
    const float2 wz0 = twz[b];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      // c2r pre-processing of positions k = b + (H/8) r (see c2r_pre)
      const float2* row = stg + (c * Z::ROWS + q) * Mzp;
      float2 v[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int k = b + Z::NB0 * r, kk = H - k;
        float2 X = below(k, Z::NB0 * r, Z::NB0 * r + Z::NB0 - 1, Mz) ? row[k] : make_float2(0.f, 0.f);
        float2 Y = below(kk, H - Z::NB0 * r - Z::NB0 + 1, H - Z::NB0 * r, Mz) ? row[kk] : make_float2(0.f, 0.f);
        if (k == 0) {
          X.y = 0.f;
          Y.y = 0.f;
        }
        Y.y = -Y.y;
        const float2 sm = cadd(X, Y), df = csub(X, Y);
        float2 w = zw_wz(wz0, r);
        w.y = -w.y;
        v[r] = cadd(sm, cmul_i(cmul(w, df)));
      }
      zw_transform<H, true>(v, xch, tws, b, mid, wl);
      if (c == 5 && grp + nwarps < ngroups) prefetch(grp + nwarps);  // every lane is past its staged reads
      // u x w (navierstokes.py:82-86) in the packed form of the real rows:
      // n0 = u1 w2 - u2 w1, n1 = u2 w0 - u0 w2, n2 = u0 w1 - u1 w0
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const float2 x = v[r];
        switch (c) {
          case 0: u0[r] = x; break;
          case 1: u1[r] = x; break;
          case 2: u2[r] = x; break;
          case 3:
            n1[r] = __fmul2_rn(u2[r], x);
            n2[r] = __fmul2_rn(u1[r], make_float2(-x.x, -x.y));
            break;
          case 4:
            n0[r] = __fmul2_rn(u2[r], make_float2(-x.x, -x.y));
            n2[r] = __ffma2_rn(u0[r], x, n2[r]);
            break;
          default:
            n0[r] = __fmul2_rn(__ffma2_rn(u1[r], x, n0[r]), make_float2(s2, s2));
            n1[r] = __fmul2_rn(__ffma2_rn(u0[r], make_float2(-x.x, -x.y), n1[r]), make_float2(s2, s2));
            n2[r] = __fmul2_rn(n2[r], make_float2(s2, s2));
            break;
        }
      }
    }
    // r2c of the three products; outputs over the first three input fields
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float2 v[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) v[r] = c == 0 ? n0[r] : (c == 1 ? n1[r] : n2[r]);
      zw_transform<H, false>(v, xch, tws, b, mid, wl);
      float2* out = a.buf + c * a.c_stride + (grp * Z::ROWS + q) * Mzp;
      const int partner = q * Z::LPR + ((Z::LPR - b) & (Z::LPR - 1));
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        // Z[H - k] of k = b + (H/8) r: lane (LPR - b) mod LPR of the row, value
        // 7 - r; for b = 0 this lane's own value (8 - r) mod 8 (Z[H] = Z[0])
        float2 t;
        t.x = __shfl_sync(0xffffffffu, v[7 - r].x, partner);
        t.y = __shfl_sync(0xffffffffu, v[7 - r].y, partner);
        const float2 zb = b == 0 ? v[(8 - r) & 7] : t;
        const int k = b + Z::NB0 * r;
        if (below(k, Z::NB0 * r, Z::NB0 * r + Z::NB0 - 1, Mzp)) {
          float2 x = make_float2(0.f, 0.f);
          if (below(k, Z::NB0 * r, Z::NB0 * r + Z::NB0 - 1, Mz)) {  // r2c_post with the 1/2 folded into s2
            float2 bc = zb;
            bc.y = -bc.y;
            const float2 E = cadd(v[r], bc), O = cmul_mi(csub(v[r], bc));
            x = cadd(E, cmul(zw_wz(wz0, r), O));
          }
          out[k] = x;
        }
      }
      // bin H (general path: Mz = H + 1) and the row padding past it
      if (!DA && b < Mzp - H) {
        float2 x = make_float2(0.f, 0.f);
        if (b == 0 && H < Mz) {
          float2 bc = v[0];
          bc.y = -bc.y;
          x = cadd(cadd(v[0], bc), cmul(twz[H], cmul_mi(csub(v[0], bc))));
        }
        out[H + b] = x;
      }
    }
  }
}

// k_zpair: k_zwarp for rows of Nz = 1024 (H = 512).  A row's half-length
// transform needs 64 lanes of 8 values, so a team of two warps owns each row,
// and its exchanges are ordered by a named barrier over the team's 64 threads
// (barrier 1 + team; 0 is __syncthreads).  The r2c post-processing partner
// Z[H - k] of lane b is lane (64 - b) mod 64, in the other warp for most b:
// the transform's outputs go through the exchange buffer instead of a
// shuffle.  Staging (one bulk TMA copy per input row, issued by the team's
// first warp on the team's mbarrier), pre-processing, u x w in registers and
// the outputs over the first three input rows are k_zwarp's.  A give-up of the
// staging wait is agreed by both warps (bar.red.and) so that they leave
// together.
constexpr int ZP_WARPS = 4;  // warps per k_zpair CTA (two teams)

// AND of v over the 64 threads of named barrier id (all must call).
__device__ __forceinline__ bool team_and(bool v, int id) {
  int r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.s32 q, %1, 0;\n\t"
      "bar.red.and.pred p, %2, 64, q;\n\t"
      "selp.s32 %0, 1, 0, p;\n\t}\n"
      : "=r"(r)
      : "r"((int)v), "r"(id)
      : "memory");
  return r != 0;
}

template <bool DA>
__global__ void __launch_bounds__(ZP_WARPS * 32, ZW_MINB) k_zpair(ZCrossArgs<float> a) {
  constexpr int H = 512, NTEAM = ZP_WARPS / 2;
  using Z = ZW<H>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) uint64_t bars[NTEAM];
  float2* tws = reinterpret_cast<float2*>(smem_raw);
  const int Mz = DA ? zw_da_mz<H>() : a.Mz;
  const int Mzp = DA ? (zw_da_mz<H>() + 7) / 8 * 8 : a.Mzp;
  auto below = [](int k, int lo, int hi, int bound) { return hi < bound ? true : (lo >= bound ? false : k < bound); };
  const int team = threadIdx.x >> 6, b = threadIdx.x & 63, lane = threadIdx.x & 31;
  const int bar_id = 1 + team;
  const ZwMid<H> mid(b);
  float2 wl[7];  // filled once the twiddle tables are in shared memory
  const int stg_slots = 6 * Mzp;
  float2* stg = tws + Z::TWS + team * (stg_slots + Z::XS);  // [field][Mzp]
  float2* xch = stg + stg_slots;
  const float2* twz = tws + Z::TWZ;
  zw_fill_twiddles<H, ZP_WARPS * 32>(tws, a.tw);
  const uint32_t mb = tma::smem_u32(&bars[team]);
  if (b == 0) tma::mbar_init(mb, 1);
  tma::fence_async_smem();
  __syncthreads();
  zw_last_twiddles<H>(wl, tws, b);

  const int wait_limit = g_z_wait_limit;
  const long long nteams = (long long)gridDim.x * NTEAM;
  const uint32_t row_bytes = (uint32_t)(Mzp * sizeof(float2));
  auto prefetch = [&](long long row) {  // the team's first warp issues the six row copies
    if (b < 32) {
      if (lane == 0) tma::mbar_expect_tx(mb, 6u * row_bytes);
      __syncwarp();
      if (lane < 6) tma::load_bytes(stg + lane * Mzp, a.buf + lane * a.c_stride + row * Mzp, row_bytes, mb);
    }
  };

  pdl_wait();
  pdl_trigger();
  long long row = (long long)blockIdx.x * NTEAM + team;
  if (row < a.nrows) prefetch(row);
  uint32_t phase = 0;
  const float s2 = 0.5f * a.scale * a.scale;  // both inverse normalisations and the r2c 1/2
  for (; row < a.nrows; row += nteams) {
    {
      const bool mine = __all_sync(0xffffffffu, tma::mbar_wait(mb, phase, wait_limit));
      const bool ok = team_and(mine, bar_id);
      phase ^= 1;
      if (!ok) {
        if (b == 0) atomicExch(&g_z_timeout, 1);
        tma::mbar_wait(mb, phase ^ 1, Z_WAIT);  // the copies in flight, once more with a limit
        return;
      }
    }
    float2 u0[8], u1[8], u2[8], n0[8], n1[8], n2[8];
    const float2 wz0 = twz[b];  // e^{-2 pi i k / Nz} of positions k = b + 64 r: zw_wz(wz0, r)
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      const float2* srow = stg + c * Mzp;
      float2 v[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int k = b + Z::NB0 * r, kk = H - k;
        float2 X = below(k, Z::NB0 * r, Z::NB0 * r + Z::NB0 - 1, Mz) ? srow[k] : make_float2(0.f, 0.f);
        float2 Y = below(kk, H - Z::NB0 * r - Z::NB0 + 1, H - Z::NB0 * r, Mz) ? srow[kk] : make_float2(0.f, 0.f);
        if (k == 0) {
          X.y = 0.f;
          Y.y = 0.f;
        }
        Y.y = -Y.y;
        const float2 sm = cadd(X, Y), df = csub(X, Y);
        float2 w = zw_wz(wz0, r);
        w.y = -w.y;
        v[r] = cadd(sm, cmul_i(cmul(w, df)));
      }
      zw_transform<H, true>(v, xch, tws, b, mid, wl, bar_id);
      // the transform's first exchange barrier put both warps past their staged reads
      if (c == 5 && row + nteams < a.nrows) prefetch(row + nteams);
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const float2 x = v[r];
        switch (c) {
          case 0: u0[r] = x; break;
          case 1: u1[r] = x; break;
          case 2: u2[r] = x; break;
          case 3:
            n1[r] = __fmul2_rn(u2[r], x);
            n2[r] = __fmul2_rn(u1[r], make_float2(-x.x, -x.y));
            break;
          case 4:
            n0[r] = __fmul2_rn(u2[r], make_float2(-x.x, -x.y));
            n2[r] = __ffma2_rn(u0[r], x, n2[r]);
            break;
          default:
            n0[r] = __fmul2_rn(__ffma2_rn(u1[r], x, n0[r]), make_float2(s2, s2));
            n1[r] = __fmul2_rn(__ffma2_rn(u0[r], make_float2(-x.x, -x.y), n1[r]), make_float2(s2, s2));
            n2[r] = __fmul2_rn(n2[r], make_float2(s2, s2));
            break;
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      float2 v[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) v[r] = c == 0 ? n0[r] : (c == 1 ? n1[r] : n2[r]);
      zw_transform<H, false>(v, xch, tws, b, mid, wl, bar_id);
      // Z[H - k] of k = b + 64 r: lane (64 - b) mod 64, value 7 - r; for b = 0
      // this lane's own value (8 - r) mod 8 (Z[H] = Z[0])
#pragma unroll
      for (int r = 0; r < 8; ++r) xch[zw_slot<H>(b + Z::NB0 * r)] = v[r];
      zw_sync<H>(bar_id);
      const int pb = (Z::LPR - b) & (Z::LPR - 1);
      float2 zb[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) zb[r] = b == 0 ? v[(8 - r) & 7] : xch[zw_slot<H>(pb + Z::NB0 * (7 - r))];
      zw_sync<H>(bar_id);  // the exchange buffer is free for the next transform
      float2* out = a.buf + c * a.c_stride + row * Mzp;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int k = b + Z::NB0 * r;
        if (below(k, Z::NB0 * r, Z::NB0 * r + Z::NB0 - 1, Mzp)) {
          float2 x = make_float2(0.f, 0.f);
          if (below(k, Z::NB0 * r, Z::NB0 * r + Z::NB0 - 1, Mz)) {  // r2c_post with the 1/2 folded into s2
            float2 bc = zb[r];
            bc.y = -bc.y;
            const float2 E = cadd(v[r], bc), O = cmul_mi(csub(v[r], bc));
            x = cadd(E, cmul(zw_wz(wz0, r), O));
          }
          out[k] = x;
        }
      }
      // bin H (general path: Mz = H + 1) and the row padding past it
      if (!DA && b < Mzp - H) {
        float2 x = make_float2(0.f, 0.f);
        if (b == 0 && H < Mz) {
          float2 bc = v[0];
          bc.y = -bc.y;
          x = cadd(cadd(v[0], bc), cmul(twz[H], cmul_mi(csub(v[0], bc))));
        }
        out[H + b] = x;
      }
    }
  }
}

// Plain z c2r / r2c (to_physical / to_spectral).  Persistent CTAs walk the
// (component, RB-row group) pairs; the rows of the next group are staged with
// cp.async while the current group is transformed (a warp per row), as in
// k_zcross.  Staged complex rows hold Mzp entries (16-byte chunks); real rows
// 2H values.
template <typename T, int H> __host__ __device__ constexpr int zreal_row_slots() {
  return z_row_cap<H>() > H ? z_row_cap<H>() : H;  // complex rows of Mzp <= z_row_cap, or real rows of H pairs
}

template <typename T, int H, int RB, int NTZ, bool C2R>
__global__ void __launch_bounds__(NTZ) k_zreal(ZRealArgs<T> a, int ncomp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  using AD = SkewAddr<skew_ld(H)>;
  constexpr int KC = z_row_cap<H>();
  constexpr int RS = zreal_row_slots<T, H>();
  V2<T>* buf = reinterpret_cast<V2<T>*>(smem_raw);
  V2<T>* tws = buf + RB * AD::LD;
  const V2<T>* twz = tws + tw_size<true>(H);
  V2<T>* raw = tws + z_tw_slots<H>();  // RB staged rows of RS slots
  fill_z_twiddles<T, H, NTZ>(tws, a.tw);
  const long long ngroups = (a.nrows + RB - 1) / RB, total = ngroups * ncomp;
  constexpr int VPC = 16 / sizeof(V2<T>);
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  constexpr int NWARP = NTZ / 32;
  // row lengths in 16-byte chunks: complex rows Mzp entries, real rows H pairs
  const int chunks = C2R ? a.Mzp / VPC : H / VPC;
  auto prefetch = [&](long long grp) {
    const long long r0 = (grp % ngroups) * RB, c = grp / ngroups;
    for (int lr = warp; lr < RB; lr += NWARP) {
      V2<T>* dst = raw + lr * RS;
      const bool in = r0 + lr < a.nrows;
      const V2<T>* src = C2R ? a.cbuf + c * a.cc_stride + (r0 + lr) * a.Mzp
                             : reinterpret_cast<const V2<T>*>(a.rbuf + c * a.rc_stride + (r0 + lr) * (2 * H));
      for (int ch = lane; ch < chunks; ch += 32) {
        if (in) cp_async16(dst + ch * VPC, src + ch * VPC);
        else
          for (int i = 0; i < VPC; ++i) dst[ch * VPC + i] = czero<T>();
      }
    }
    cp_async_commit();
  };
  long long grp = blockIdx.x;
  if (grp < total) prefetch(grp);
  for (; grp < total; grp += gridDim.x) {
    const long long row0 = (grp % ngroups) * RB, c = grp / ngroups;
    cp_async_wait_all();
    __syncthreads();
    const long long nxt = grp + gridDim.x;
    if constexpr (C2R) {
      fft_ip<T, H, RB, NTZ, AD, true>(
          buf, tws, [&](int k, int lr) { return c2r_pre<T>(raw + lr * RS, k, H, a.Mz, twz); },
          [&](int m, int lr, V2<T> v) {
            if (row0 + lr < a.nrows)
              reinterpret_cast<V2<T>*>(a.rbuf + c * a.rc_stride + (row0 + lr) * (2 * H))[m] = cscale(v, a.scale);
          },
          [&]() {
            if (nxt < total) prefetch(nxt);
          });
    } else {
      fft_ip<T, H, RB, NTZ, AD, false>(
          buf, tws, [&](int m, int lr) { return raw[lr * RS + m]; },
          [&](int k, int lr, V2<T> v) { buf[AD::at(k, lr)] = v; },
          [&]() {
            if (nxt < total) prefetch(nxt);
          });
      for (int e = threadIdx.x; e < RB * KC; e += NTZ) {
        const int lr = e / KC, k = e % KC;
        if (row0 + lr < a.nrows && k < a.Mzp) {
          V2<T> v = czero<T>();
          if (k < a.Mz) v = r2c_post<T>([&](int i) { return buf[AD::at(i, lr)]; }, k, H, twz);
          a.cbuf[c * a.cc_stride + (row0 + lr) * a.Mzp + k] = v;
        }
      }
      __syncthreads();  // buf is rewritten by the next group
    }
  }
  cp_async_wait_all();
}

// r2c with one CTA per (RB-row group, component): many small CTAs in flight
// hide the latency of the direct row loads, which measured faster than the
// persistent staged form for the r2c direction.
template <typename T, int H, int RB, int NTZ>
__global__ void __launch_bounds__(NTZ) k_zr2c(ZRealArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  using AD = SkewAddr<skew_ld(H)>;
  constexpr int KC = z_row_cap<H>();
  V2<T>* buf = reinterpret_cast<V2<T>*>(smem_raw);
  V2<T>* tws = buf + RB * AD::LD;
  const V2<T>* twz = tws + tw_size<true>(H);
  fill_z_twiddles<T, H, NTZ>(tws, a.tw);
  const long long row0 = (long long)blockIdx.x * RB;
  const long long c = blockIdx.y;
  fft_ip<T, H, RB, NTZ, AD, false>(
      buf, tws,
      [&](int m, int lr) {
        if (row0 + lr >= a.nrows) return czero<T>();
        return reinterpret_cast<const V2<T>*>(a.rbuf + c * a.rc_stride + (row0 + lr) * (2 * H))[m];
      },
      [&](int k, int lr, V2<T> v) { buf[AD::at(k, lr)] = v; });
  for (int e = threadIdx.x; e < RB * KC; e += NTZ) {
    const int lr = e / KC, k = e % KC;
    if (row0 + lr < a.nrows && k < a.Mzp) {
      V2<T> v = czero<T>();
      if (k < a.Mz) v = r2c_post<T>([&](int i) { return buf[AD::at(i, lr)]; }, k, H, twz);
      a.cbuf[c * a.cc_stride + (row0 + lr) * a.Mzp + k] = v;
    }
  }
}

// Polls of the row-group wait of k_zcross on the current device (polls < 0:
// the default).
cudaError_t set_z_wait_limit(int polls) {
  const int v = polls < 0 ? Z_WAIT : polls;
  return cudaMemcpyToSymbol(g_z_wait_limit, &v, sizeof(int));
}

// Read and clear the flag a TMA wait of k_zcross sets when it gives up.
cudaError_t take_z_timeout(int* flag) {
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_z_timeout, sizeof(int));
  if (e != cudaSuccess) return e;
  *flag = v;
  const int zero = 0;
  return v ? cudaMemcpyToSymbol(g_z_timeout, &zero, sizeof(int)) : cudaSuccess;
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

template <typename T, int H> constexpr size_t zr2c_smem() {
  return sizeof(V2<T>) * (z_rows_per_block<H>() * skew_ld(H) + z_tw_slots<H>());
}
template <typename T, int H> constexpr size_t zreal_smem() {
  return sizeof(V2<T>) * (z_rows_per_block<H>() * (skew_ld(H) + zreal_row_slots<T, H>()) + z_tw_slots<H>());
}

template <typename T, int HH, int RB, int NTZ, int MINB> cudaError_t launch_zcross_v(const ZCrossArgs<T>& a, cudaStream_t st) {
  static PerDevice ready, cache;
  const size_t smem = sizeof(V2<T>) * (6 * RB * skew_ld(HH) + z_tw_slots<HH>() + 6 * RB * z_row_cap<HH>());
  cudaError_t e = once_per_device(ready, [&] {
    cudaError_t r = cudaFuncSetAttribute(k_zcross<T, HH, RB, NTZ, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (r != cudaSuccess) return r;
    return cudaFuncSetAttribute(k_zcross<T, HH, RB, NTZ, MINB>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared);
  });
  if (e != cudaSuccess) return e;
  const int nb = resident_grid(k_zcross<T, HH, RB, NTZ, MINB>, NTZ, smem, (a.nrows + RB - 1) / RB, cache);
  return launch_pdl(k_zcross<T, HH, RB, NTZ, MINB>, nb, NTZ, smem, st, a);
}

// Warps per k_zwarp CTA.
constexpr int ZW_WARPS = 4;

template <int HH> size_t zwarp_smem(int Mzp) {
  using Z = ZW<HH>;
  return sizeof(float2) * (Z::TWS + (size_t)ZW_WARPS * (6 * Z::ROWS * Mzp + Z::ROWS * Z::XS));
}

template <int HH, bool DA> cudaError_t launch_zwarp_v(const ZCrossArgs<float>& a, cudaStream_t st) {
  static PerDevice ready, cache;
  // the opt-in covers the largest staging rows (Mzp = H + 8)
  const size_t smax = zwarp_smem<HH>(HH + 8);
  cudaError_t e = once_per_device(ready, [&] {
    cudaError_t r = cudaFuncSetAttribute(k_zwarp<HH, ZW_WARPS, DA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smax);
    if (r != cudaSuccess) return r;
    return cudaFuncSetAttribute(k_zwarp<HH, ZW_WARPS, DA>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared);
  });
  if (e != cudaSuccess) return e;
  const size_t smem = zwarp_smem<HH>(a.Mzp);
  const long long groups = a.nrows / ZW<HH>::ROWS;
  const int nb =
      resident_grid(k_zwarp<HH, ZW_WARPS, DA>, ZW_WARPS * 32, smax, (groups + ZW_WARPS - 1) / ZW_WARPS, cache);
  return launch_pdl(k_zwarp<HH, ZW_WARPS, DA>, nb, ZW_WARPS * 32, smem, st, a);
}

template <int HH> cudaError_t launch_zwarp(const ZCrossArgs<float>& a, cudaStream_t st) {
  const bool da = a.Mz == zw_da_mz<HH>() && a.Mzp == (zw_da_mz<HH>() + 7) / 8 * 8;
  return da ? launch_zwarp_v<HH, true>(a, st) : launch_zwarp_v<HH, false>(a, st);
}

template <bool DA> cudaError_t launch_zpair_v(const ZCrossArgs<float>& a, cudaStream_t st) {
  static PerDevice ready, cache;
  using Z = ZW<512>;
  constexpr int NTEAM = ZP_WARPS / 2;
  auto smem_of = [](int Mzp) { return sizeof(float2) * (Z::TWS + (size_t)NTEAM * (6 * Mzp + Z::XS)); };
  const size_t smax = smem_of(512 + 8);  // the opt-in covers the largest staging rows
  cudaError_t e = once_per_device(ready, [&] {
    cudaError_t r = cudaFuncSetAttribute(k_zpair<DA>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax);
    if (r != cudaSuccess) return r;
    return cudaFuncSetAttribute(k_zpair<DA>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared);
  });
  if (e != cudaSuccess) return e;
  const int nb = resident_grid(k_zpair<DA>, ZP_WARPS * 32, smax, (a.nrows + NTEAM - 1) / NTEAM, cache);
  return launch_pdl(k_zpair<DA>, nb, ZP_WARPS * 32, smem_of(a.Mzp), st, a);
}

cudaError_t launch_zpair(const ZCrossArgs<float>& a, cudaStream_t st) {
  const bool da = a.Mz == zw_da_mz<512>() && a.Mzp == (zw_da_mz<512>() + 7) / 8 * 8;
  return da ? launch_zpair_v<true>(a, st) : launch_zpair_v<false>(a, st);
}

// float32 rows of Nz = 64 ... 1024 (whole row groups, staging rows of at most
// H + 8 entries) take the warp-resident kernels (a warp pair per row at Nz =
// 1024); every other case k_zcross.
template <typename T> bool use_zwarp(int H, const ZCrossArgs<T>& a) {
  if (!std::is_same<T, float>::value || !(H == 32 || H == 64 || H == 128 || H == 256 || H == 512)) return false;
  const int rows = H <= 256 ? 256 / H : 1;
  return a.nrows % rows == 0 && a.Mzp % 8 == 0 && a.Mzp <= H + 8 && a.Mz <= a.Mzp;
}

template <typename T> cudaError_t launch_zcross(int H, const ZCrossArgs<T>& a, cudaStream_t st) {
  if constexpr (std::is_same<T, float>::value) {
    if (use_zwarp(H, a)) {
      if (H == 32) return launch_zwarp<32>(a, st);
      if (H == 64) return launch_zwarp<64>(a, st);
      if (H == 128) return launch_zwarp<128>(a, st);
      if (H == 256) return launch_zwarp<256>(a, st);
      return launch_zpair(a, st);
    }
  }
  return dispatch_half(H, [&](auto hh) {
    constexpr int HH = decltype(hh)::value;
    return launch_zcross_v<T, HH, z_rows_per_block<HH>(), z_threads<HH>(), 4>(a, st);
  });
}

template <int HH> size_t zles_smem() {
  using AD = SkewAddr<skew_ld(HH)>;
  constexpr int RB = 128 / (2 * HH);
  return (sizeof(mlp::InferSmem) + 127) / 128 * 128 +
         sizeof(float2) * (12 * RB * AD::LD + z_tw_slots<HH>() + 12 * RB * z_row_cap<HH>());
}

template <int HH> cudaError_t launch_zles_v(const ZLesArgs& a, cudaStream_t st) {
  static PerDevice ready, cache;
  constexpr int RB = 128 / (2 * HH);
  const size_t smem = zles_smem<HH>();
  cudaError_t e = once_per_device(ready, [&] {
    cudaError_t r = cudaFuncSetAttribute(k_zles<HH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (r != cudaSuccess) return r;
    return cudaFuncSetAttribute(k_zles<HH>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                cudaSharedmemCarveoutMaxShared);
  });
  if (e != cudaSuccess) return e;
  // resident CTAs from the SM's shared memory and registers (the occupancy
  // query counts one CTA per SM for kernels that allocate tensor memory), at
  // most 8 per SM (8 x 64 TMEM columns)
  std::atomic<int>* slot = cache.here();
  int wave = slot ? slot->load(std::memory_order_relaxed) : 0;
  if (wave == 0) {
    int dev = 0, sms = 0, smem_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess)
      return e;
    int regs_sm = 0;
    cudaFuncAttributes fa{};
    if ((e = cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev)) != cudaSuccess) return e;
    if ((e = cudaFuncGetAttributes(&fa, k_zles<HH>)) != cudaSuccess) return e;
    const int by_regs = regs_sm / (128 * ((std::max(fa.numRegs, 1) + 7) / 8 * 8));
    const int per_sm = std::max(1, std::min(std::min((int)(smem_sm / (smem + 1024 + 64)), by_regs), 8));
    wave = per_sm * std::max(sms, 1);
    if (slot) slot->store(wave, std::memory_order_relaxed);
  }
  const int groups = (a.nrows + RB - 1) / RB;
  return launch_pdl(k_zles<HH>, std::max(1, std::min(groups, wave)), 128, smem, st, a);
}

bool zles_supported(int Nz) { return Nz == 32 || Nz == 64 || Nz == 128; }

cudaError_t launch_zles(int H, const ZLesArgs& a, cudaStream_t st) {
  if (a.Mzp % 8 || a.Mzp > (H + 1 + 7) / 8 * 8) return cudaErrorInvalidValue;
  if (H == 16) return launch_zles_v<16>(a, st);
  if (H == 32) return launch_zles_v<32>(a, st);
  if (H == 64) return launch_zles_v<64>(a, st);
  return cudaErrorInvalidValue;
}

template <typename T, bool C2R> cudaError_t launch_zreal(int H, const ZRealArgs<T>& a, int ncomp, cudaStream_t st) {
  if (a.Mzp % 8 || ((uintptr_t)a.cbuf % 16) || ((uintptr_t)a.rbuf % 16)) return cudaErrorInvalidValue;
  return dispatch_half(H, [&](auto hh) {
    constexpr int HH = decltype(hh)::value;
    constexpr int RB = z_rows_per_block<HH>(), NTZ = z_threads<HH>();
    if (a.Mzp > z_row_cap<HH>()) return cudaErrorInvalidValue;
    static PerDevice cache;
    const long long work = (a.nrows + RB - 1) / RB * ncomp;
    const int grid = resident_grid(k_zreal<T, HH, RB, NTZ, C2R>, NTZ, zreal_smem<T, HH>(), work, cache);
    k_zreal<T, HH, RB, NTZ, C2R><<<grid, NTZ, zreal_smem<T, HH>(), st>>>(a, ncomp);
    return cudaGetLastError();
  });
}
template <typename T> cudaError_t launch_zc2r(int H, const ZRealArgs<T>& a, int ncomp, cudaStream_t st) {
  return launch_zreal<T, true>(H, a, ncomp, st);
}
template <typename T> cudaError_t launch_zr2c(int H, const ZRealArgs<T>& a, int ncomp, cudaStream_t st) {
  return dispatch_half(H, [&](auto hh) {
    constexpr int HH = decltype(hh)::value;
    constexpr int RB = z_rows_per_block<HH>();
    dim3 grid((a.nrows + RB - 1) / RB, ncomp);
    k_zr2c<T, HH, RB, z_threads<HH>()><<<grid, z_threads<HH>(), zr2c_smem<T, HH>(), st>>>(a);
    return cudaGetLastError();
  });
}

template <typename T> cudaError_t prepare_axis_kernels(int Nx);

template <typename K> cudaError_t max_smem(K kernel, int bytes) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
}

template <typename T> cudaError_t prepare_fft_kernels(int Nx, int Ny, int Nz) {
  cudaError_t e = prepare_axis_kernels<T>(Nx);
  if (e != cudaSuccess) return e;
  if (Ny != Nx && (e = prepare_axis_kernels<T>(Ny)) != cudaSuccess) return e;
  return dispatch_half(Nz / 2, [&](auto hh) {
    constexpr int HH = decltype(hh)::value;
    constexpr int RB = z_rows_per_block<HH>();
    constexpr int NTZ = z_threads<HH>();
    cudaError_t r = max_smem(k_zreal<T, HH, RB, NTZ, true>, (int)zreal_smem<T, HH>());
    if (r != cudaSuccess) return r;
    return max_smem(k_zr2c<T, HH, RB, NTZ>, (int)zr2c_smem<T, HH>());
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
