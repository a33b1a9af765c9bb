// Pointwise MLP of the learned subgrid-stress closure on the fifth-generation
// tensor cores: 9 -> 64 -> 64 -> 64 -> 6, GELU between layers, bf16 weights
// and activations, float32 accumulation in TMEM.
//
// One persistent CTA of 128 threads works on 128-point tiles; thread t owns
// point t of the tile (its TMEM lane).  The weight operands stay in shared
// memory in the K-major core-matrix layout (tc_common.cuh).  Per tile:
//   forward   z1 = [x, 0, 1] W1 (bias in row 15), a_l = gelu(z_l),
//             z_l = a_{l-1} W_l + b_l (l = 2, 3), y = a3 W4 + b4;
//   training  dy = 2 (y - tau) / (P * 6) (the MSE loss), then
//             da_{l-1} = dz_l W_l^T, dz_{l-1} = da_{l-1} * gelu'(z_{l-1}),
// the pre-activations z1..z3 staying in TMEM for gelu'.  The activations
// a_{l-1} (with a ones row for the bias) and the dz_l are written feature-major
// (aT[f][p], dzT[f][p], bf16) for the weight-gradient GEMMs
// dW_l = a_{l-1}^T dz_l, which run on the same tensor cores (k_tcgemm).
//
// Two instantiations: TRAIN (forward + backward: the backward weights W_2..4
// resident too, z1..z3 kept in 256 TMEM columns, two CTAs per SM) and the
// inference one (forward weights only, one activation buffer, every layer's
// accumulator in the same 64 TMEM columns: about half the shared memory, so
// more CTAs per SM hide the per-layer MMA round trip).
#include <cuda_bf16.h>

#include <algorithm>

#include "kernels.h"
#include "mlp_core.cuh"
#include "tc_common.cuh"

namespace hit {

using namespace mlp;

namespace {
constexpr int MLP_WAIT = 1 << 22;
}  // namespace

template <bool TRAIN> struct MlpSmem {
  unsigned char w1t[64 * 16 * 2], w2t[64 * 64 * 2], w3t[64 * 64 * 2], w4t[16 * 64 * 2];
  // backward operands (training only)
  unsigned char w4[TRAIN ? 64 * 16 * 2 : 16], w3[TRAIN ? 64 * 64 * 2 : 16], w2[TRAIN ? 64 * 64 * 2 : 16];
  unsigned char w1[TRAIN ? 16 * 64 * 2 : 16];  // backward layer 1 (input gradient, vector-Jacobian mode)
  unsigned char x0[128 * 16 * 2];                   // a0, later dz4
  unsigned char buf[TRAIN ? 2 : 1][128 * 64 * 2];  // activations / gradients (ping-pong when training)
  float b2[64], b3[64], b4[16];
  double red[4];
  uint64_t mbar;
  uint32_t tslot;
};

template <bool TRAIN>
__global__ void __launch_bounds__(128) k_mlp(MlpArgs a) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  MlpSmem<TRAIN>& S = *reinterpret_cast<MlpSmem<TRAIN>*>(smem_raw);
  // TMEM columns of the layer accumulators: z1..z3 kept for the backward when
  // training; one 64-column accumulator reused by every layer otherwise
  constexpr uint32_t C1 = 0, C2 = TRAIN ? 64 : 0, C3 = TRAIN ? 128 : 0, C4 = TRAIN ? 192 : 0;
  constexpr uint32_t NCOL = TRAIN ? 256 : 64;
  constexpr int B1 = TRAIN ? 1 : 0;  // buffer of the second layer's output
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t mb = tc::smem_u32(&S.mbar);
  // weights and biases (resident for all tiles)
  load_kmajor(S.w1t, a.w1t, 64, 16);
  load_kmajor(S.w2t, a.w2t, 64, 64);
  load_kmajor(S.w3t, a.w3t, 64, 64);
  load_kmajor(S.w4t, a.w4t, 16, 64);
  constexpr bool train = TRAIN;
  if constexpr (TRAIN) {
    load_kmajor(S.w4, a.w4, 64, 16);
    load_kmajor(S.w3, a.w3, 64, 64);
    load_kmajor(S.w2, a.w2, 64, 64);
    if (a.xbar) load_kmajor(S.w1, a.w1, 16, 64);
  }
  for (int i = tid; i < 64; i += 128) {
    S.b2[i] = a.b2[i];
    S.b3[i] = a.b3[i];
  }
  if (tid < 16) S.b4[tid] = a.b4[tid];
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(&S.tslot), NCOL);
  if (tid == 0) tc::mbar_init(mb, 1);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = S.tslot;
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's TMEM lanes
  uint32_t phase = 0;
  bool ok = true;
  double loss = 0.0;
  const uint32_t id64 = tc::idesc_bf16(128, 64), id16 = tc::idesc_bf16(128, 16);

  // D[col0..] = A (KC columns, k_steps steps) * B^T; every thread waits.
  auto mma = [&](uint32_t col0, const unsigned char* A, int KCa, const unsigned char* B, int KCb, int steps,
                 uint32_t idesc) {
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
      const uint32_t a0 = tc::smem_u32(A), b0 = tc::smem_u32(B);
      for (int s = 0; s < steps; ++s)
        tc::mma_bf16(tmem + col0, tc::smem_desc(a0 + 256 * s, 128, KCa * 16), tc::smem_desc(b0 + 256 * s, 128, KCb * 16),
                     idesc, s > 0);
      tc::commit(mb);
    }
    ok = __syncthreads_and(ok && tc::mbar_wait(mb, phase, MLP_WAIT)) != 0;  // block-uniform
    phase ^= 1;
    tc::fence_after_sync();
  };
  auto ld64 = [&](uint32_t col0, float (&v)[64]) {
#pragma unroll
    for (int c = 0; c < 64; c += 16) {
      float t[16];
      tc::tmem_ld16(lane_base + col0 + c, t);
#pragma unroll
      for (int i = 0; i < 16; ++i) v[c + i] = t[i];
    }
  };
  // feature-major bf16 row f of an [F][P] array
  auto put_t = [&](__nv_bfloat16* dst, int f, long long p, float v) { dst[(long long)f * a.P + p] = __float2bfloat16_rn(v); };

  for (int tile = blockIdx.x; tile * 128 < a.P && ok; tile += gridDim.x) {
    const long long p = (long long)tile * 128 + tid;
    const bool in = p < a.P;
    // ---- forward ----
    float v[64];
    {
      float x[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) x[i] = 0.f;
      if (in) {
#pragma unroll
        for (int i = 0; i < 9; ++i) x[i] = a.x[i * a.x_sf + p * a.x_sp];
      }
      x[15] = in ? 1.f : 0.f;  // bias input of layer 1
      store_row<16>(S.x0, tid, x, 16);
      if (train && in) {
#pragma unroll
        for (int i = 0; i < 16; ++i) put_t(a.aT0, i, p, x[i]);
      }
    }
    // (a layer's accumulator columns and input buffer are rewritten only after
    // the MMA that reads them has completed and every thread has loaded them)
    mma(C1, S.x0, 16, S.w1t, 16, 1, id64);
    ld64(C1, v);
#pragma unroll
    for (int i = 0; i < 64; ++i) v[i] = gelu(v[i]);
    store_row<64>(S.buf[0], tid, v, 64);
    if (train && in) {
#pragma unroll 8
      for (int i = 0; i < 64; ++i) put_t(a.aT1, i, p, v[i]);
      put_t(a.aT1, 64, p, 1.f);
    }
    mma(C2, S.buf[0], 64, S.w2t, 64, 4, id64);
    ld64(C2, v);
#pragma unroll
    for (int i = 0; i < 64; ++i) v[i] = gelu(v[i] + S.b2[i]);
    store_row<64>(S.buf[B1], tid, v, 64);
    if (train && in) {
#pragma unroll 8
      for (int i = 0; i < 64; ++i) put_t(a.aT2, i, p, v[i]);
      put_t(a.aT2, 64, p, 1.f);
    }
    mma(C3, S.buf[B1], 64, S.w3t, 64, 4, id64);
    ld64(C3, v);
#pragma unroll
    for (int i = 0; i < 64; ++i) v[i] = gelu(v[i] + S.b3[i]);
    store_row<64>(S.buf[0], tid, v, 64);
    if (train && in) {
#pragma unroll 8
      for (int i = 0; i < 64; ++i) put_t(a.aT3, i, p, v[i]);
      put_t(a.aT3, 64, p, 1.f);
    }
    mma(C4, S.buf[0], 64, S.w4t, 64, 4, id16);
    float y[16];
    tc::tmem_ld16(lane_base + C4, y);
#pragma unroll
    for (int i = 0; i < 6; ++i) y[i] += S.b4[i];
    if (in && a.y) {
#pragma unroll
      for (int i = 0; i < 6; ++i) a.y[i * a.y_sf + p * a.y_sp] = y[i];
    }
    if constexpr (TRAIN) {
      // ---- backward ----
      float dz[16];
  #pragma unroll
      for (int i = 0; i < 16; ++i) dz[i] = 0.f;
      if (in && a.ybar) {  // vector-Jacobian mode: the upstream dL/dy
  #pragma unroll
        for (int i = 0; i < 6; ++i) dz[i] = a.ybar[i * a.yb_sf + p * a.yb_sp];
      } else if (in) {
  #pragma unroll
        for (int i = 0; i < 6; ++i) {
          const float r = y[i] - a.tau[p * 6 + i];
          loss += (double)r * r;
          dz[i] = 2.f * r * a.inv_count;
        }
      }
      store_row<16>(S.x0, tid, dz, 16);
      if (in) {
  #pragma unroll
        for (int i = 0; i < 16; ++i) put_t(a.dzT4, i, p, dz[i]);
      }
      // dz_l from da_l (TMEM cols 192..255) and z_l (cols zcol..)
      auto back = [&](uint32_t zcol, unsigned char* dst, __nv_bfloat16* dzT, const float* bias) {
        float da[64], z[64];
        ld64(192, da);
        ld64(zcol, z);
  #pragma unroll
        for (int i = 0; i < 64; ++i) da[i] *= gelu_d(z[i] + (bias ? bias[i] : 0.f));
        if (dst) store_row<64>(dst, tid, da, 64);
        if (in) {
  #pragma unroll 8
          for (int i = 0; i < 64; ++i) put_t(dzT, i, p, da[i]);
        }
      };
      mma(192, S.x0, 16, S.w4, 16, 1, id64);  // da3 = dz4 W4^T
      back(128, S.buf[1], a.dzT3, S.b3);
      mma(192, S.buf[1], 64, S.w3, 64, 4, id64);  // da2 = dz3 W3^T
      back(64, S.buf[0], a.dzT2, S.b2);
      mma(192, S.buf[0], 64, S.w2, 64, 4, id64);  // da1 = dz2 W2^T
      back(0, a.xbar ? S.buf[1] : nullptr, a.dzT1, nullptr);
      if (a.xbar) {  // dx = dz1 W1 (TMEM columns 0..15, free once z1 is read)
        mma(0, S.buf[1], 64, S.w1, 64, 4, id16);
        float dx[16];
        tc::tmem_ld16(lane_base, dx);
        if (in) {
  #pragma unroll
          for (int i = 0; i < 9; ++i) a.xbar[i * a.x_sf + p * a.x_sp] = dx[i];
        }
      }
    }
  }
  if (!ok && tid == 0) atomicExch(a.err, 1);
  if (train && a.loss) {  // per-CTA partial of sum (y - tau)^2
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if (lane == 0) S.red[warp] = loss;
    __syncthreads();
    if (tid == 0) a.loss[blockIdx.x] = S.red[0] + S.red[1] + S.red[2] + S.red[3];
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tmem, NCOL);
}

size_t mlp_smem_bytes() { return sizeof(MlpSmem<true>); }

// Training pass when a.tau is set, else inference.  grid <= 0: one resident
// wave of CTAs (at most 8 per SM: 8 x 64 TMEM columns fill the SM's 512), or
// -k: k CTAs per SM (a lighter footprint next to other work on the GPU).
cudaError_t launch_mlp(const MlpArgs& a, int grid, cudaStream_t st) {
  // per device: the attribute set-up of each instantiation, and the
  // inference wave (CTAs per SM, and that times the SM count)
  static PerDevice ready[2], wave_of, per_sm_of;
  const bool train = a.tau != nullptr;
  const int smem = train ? (int)sizeof(MlpSmem<true>) : (int)sizeof(MlpSmem<false>);
  cudaError_t e = once_per_device(ready[train], [&] {
    // the largest shared-memory carveout, so that the occupancy below (and the
    // launch) can place several CTAs per SM
    auto setup = [&](auto kernel) {
      cudaError_t r = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
      if (r != cudaSuccess) return r;
      return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  (int)cudaSharedmemCarveoutMaxShared);
    };
    return train ? setup(k_mlp<true>) : setup(k_mlp<false>);
  });
  if (e != cudaSuccess) return e;
  int wave = 0, per_sm_wave = 1;
  if (!train) {
    std::atomic<int>* ws = wave_of.here();
    std::atomic<int>* ps = per_sm_of.here();
    wave = ws ? ws->load(std::memory_order_relaxed) : 0;
    per_sm_wave = ps ? ps->load(std::memory_order_relaxed) : 0;
    if (wave == 0 || per_sm_wave == 0) {
      // CTAs per SM from the SM's shared memory and registers (1 KB of
      // shared memory per CTA is the driver's)
      int dev = 0, sms = 0, smem_sm = 0, regs_sm = 0;
      cudaFuncAttributes fa{};
      if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
      if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
      if ((e = cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess)
        return e;
      if ((e = cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev)) != cudaSuccess)
        return e;
      if ((e = cudaFuncGetAttributes(&fa, k_mlp<false>)) != cudaSuccess) return e;
      const int by_smem = smem_sm / (smem + 1024);
      const int by_regs = regs_sm / (128 * ((std::max(fa.numRegs, 1) + 7) / 8 * 8));
      per_sm_wave = std::max(1, std::min(std::min(by_smem, by_regs), 8));
      wave = per_sm_wave * sms;
      if (ps) ps->store(per_sm_wave, std::memory_order_relaxed);
      if (ws) ws->store(wave, std::memory_order_relaxed);
    }
  }
  const long long tiles = (a.P + 127) / 128;
  if (grid < 0 && !train) grid = (int)std::min<long long>(tiles, std::min(-grid * (wave / per_sm_wave), wave));
  if (grid <= 0) grid = (int)std::min<long long>(tiles, train ? 2 * 148 : wave);
  if (train) k_mlp<true><<<grid, 128, smem, st>>>(a);
  else k_mlp<false><<<grid, 128, smem, st>>>(a);
  return cudaGetLastError();
}

}  // namespace hit
