// Device pieces of the closure MLP (9 -> 64 -> 64 -> 64 -> 6, GELU, bf16
// operands, float32 accumulation in TMEM) shared by the standalone MLP kernel
// (k_mlp.cu) and the fused LES z pass (k_zles.cu): the activation, the
// K-major operand layout copies, and one inference pass over a 128-point tile.
#pragma once

#include <cuda_bf16.h>

#include "kernels.h"
#include "tc_common.cuh"

namespace hit {
namespace mlp {

// GELU in its tanh form (Hendrycks and Gimpel, 2016),
//   gelu(x) = x/2 (1 + tanh(u)),  u = sqrt(2/pi) (x + 0.044715 x^3),
// with the hardware tanh (tanh.approx.f32, relative error about 2^-11, below
// the bf16 rounding the activations get next), and its exact derivative
//   gelu'(x) = (1 + t)/2 + x/2 (1 - t^2) sqrt(2/pi) (1 + 3 * 0.044715 x^2).
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu(float x) {
  const float t = tanh_hw(x * fmaf(0.035677408136300125f, x * x, 0.7978845608028654f));
  const float h = 0.5f * x;
  return fmaf(h, t, h);
}
__device__ __forceinline__ float gelu_d(float x) {
  const float t = tanh_hw(x * fmaf(0.035677408136300125f, x * x, 0.7978845608028654f));
  const float du = fmaf(0.10703222440890037f, x * x, 0.7978845608028654f);
  return fmaf(0.5f * x * fmaf(-t, t, 1.f), du, 0.5f * (1.f + t));
}

// Copy a row-major bf16 matrix [R][KC] into the K-major core-matrix layout.
__device__ __forceinline__ void load_kmajor(unsigned char* dst, const __nv_bfloat16* __restrict__ src, int R, int KC) {
  for (int e = threadIdx.x; e < R * (KC / 8); e += blockDim.x) {
    const int r = e / (KC / 8), c8 = e % (KC / 8);
    *reinterpret_cast<uint4*>(dst + tc::kmajor_off(r, c8 * 8, KC)) =
        *reinterpret_cast<const uint4*>(src + (long long)r * KC + c8 * 8);
  }
}

// This thread's row (point) of a K-major tile with KC columns from n floats
// (columns past n are zero).
template <int KC>
__device__ __forceinline__ void store_row(unsigned char* tile, int row, const float* v, int n) {
#pragma unroll
  for (int c8 = 0; c8 < KC / 8; ++c8) {
    __align__(16) __nv_bfloat16 h[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) h[i] = __float2bfloat16_rn(c8 * 8 + i < n ? v[c8 * 8 + i] : 0.f);
    *reinterpret_cast<uint4*>(tile + tc::kmajor_off(row, c8 * 8, KC)) = *reinterpret_cast<const uint4*>(h);
  }
}

// Shared memory of an inference pass: the forward weight operands (K-major
// core-matrix layout, layer 1 with its bias folded into input column 15), the
// layer input tile and one activation tile, the biases of layers 2-4, the
// MMA completion barrier and the TMEM base.
struct InferSmem {
  unsigned char w1t[64 * 16 * 2], w2t[64 * 64 * 2], w3t[64 * 64 * 2], w4t[16 * 64 * 2];
  unsigned char x0[128 * 16 * 2];
  unsigned char buf[128 * 64 * 2];
  float b2[64], b3[64], b4[16];
  uint64_t mbar;
  uint32_t tslot;
};
constexpr uint32_t INFER_COLS = 64;  // TMEM columns: one 64-column accumulator for every layer

// Load the weights and biases, initialise the barrier and allocate TMEM
// (all 128 threads of the CTA; warp 0 allocates).  The caller synchronises
// (__syncthreads with the tcgen05 fences) before the first tile.
__device__ __forceinline__ void infer_setup(InferSmem& S, const __nv_bfloat16* w1t, const __nv_bfloat16* w2t,
                                            const __nv_bfloat16* w3t, const __nv_bfloat16* w4t, const float* b2,
                                            const float* b3, const float* b4) {
  load_kmajor(S.w1t, w1t, 64, 16);
  load_kmajor(S.w2t, w2t, 64, 64);
  load_kmajor(S.w3t, w3t, 64, 64);
  load_kmajor(S.w4t, w4t, 16, 64);
  for (int i = threadIdx.x; i < 64; i += blockDim.x) {
    S.b2[i] = b2[i];
    S.b3[i] = b3[i];
  }
  if (threadIdx.x < 16) S.b4[threadIdx.x] = b4[threadIdx.x];
  if (threadIdx.x < 32) tc::tmem_alloc(tc::smem_u32(&S.tslot), INFER_COLS);
  if (threadIdx.x == 0) tc::mbar_init(tc::smem_u32(&S.mbar), 1);
  tc::fence_async_smem();
}

// One forward pass over a 128-point tile: thread t (of 128) gives the 9
// inputs of point t and receives its 6 outputs.  Every thread calls it; the
// MMAs are issued by thread 0 and their completion waits are bounded
// (ok becomes false, block-uniformly, when one gives up; the outputs are then
// not meaningful).  phase: the barrier's phase bit, carried across calls.
__device__ __forceinline__ void infer_tile(InferSmem& S, const float (&x9)[9], float (&y6)[6], uint32_t& phase,
                                           bool& ok, int wait_limit) {
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t tmem = S.tslot;
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
  const uint32_t mb = tc::smem_u32(&S.mbar);
  const uint32_t id64 = tc::idesc_bf16(128, 64), id16 = tc::idesc_bf16(128, 16);
  auto mma = [&](const unsigned char* A, int KCa, const unsigned char* B, int KCb, int steps, uint32_t idesc) {
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0 && ok) {  // after a wait gave up, nothing more is issued
      const uint32_t a0 = tc::smem_u32(A), b0 = tc::smem_u32(B);
      for (int s = 0; s < steps; ++s)
        tc::mma_bf16(tmem, tc::smem_desc(a0 + 256 * s, 128, KCa * 16), tc::smem_desc(b0 + 256 * s, 128, KCb * 16),
                     idesc, s > 0);
      tc::commit(mb);
    }
    ok = __syncthreads_and(ok && tc::mbar_wait(mb, phase, wait_limit)) != 0;
    phase ^= 1;
    tc::fence_after_sync();
  };
  // the 64 accumulator columns of this thread's point, 16 at a time: plus
  // the bias, GELU, rounded to bf16 into the next layer's input tile (a live
  // set of 16 values instead of 64)
  auto act64 = [&](const float* bias) {
#pragma unroll
    for (int c = 0; c < 64; c += 16) {
      float t[16];
      tc::tmem_ld16(lane_base + c, t);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        __align__(16) __nv_bfloat16 q[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) q[i] = __float2bfloat16_rn(gelu(t[8 * h + i] + (bias ? bias[c + 8 * h + i] : 0.f)));
        *reinterpret_cast<uint4*>(S.buf + tc::kmajor_off(tid, c + 8 * h, 64)) = *reinterpret_cast<const uint4*>(q);
      }
    }
  };
  {
    float x[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) x[i] = i < 9 ? x9[i] : 0.f;
    x[15] = 1.f;  // bias input of layer 1
    store_row<16>(S.x0, tid, x, 16);
  }
  // (a layer's input tile is rewritten only after the MMA that reads it has
  // completed: mma() returns after its completion wait)
  mma(S.x0, 16, S.w1t, 16, 1, id64);
  act64(nullptr);
  mma(S.buf, 64, S.w2t, 64, 4, id64);
  act64(S.b2);
  mma(S.buf, 64, S.w3t, 64, 4, id64);
  act64(S.b3);
  mma(S.buf, 64, S.w4t, 64, 4, id16);
  float y[16];
  tc::tmem_ld16(lane_base, y);
#pragma unroll
  for (int i = 0; i < 6; ++i) y6[i] = y[i] + S.b4[i];
}

// Free the TMEM of infer_setup (all threads; warp 0 deallocates).
__device__ __forceinline__ void infer_teardown(InferSmem& S) {
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (threadIdx.x < 32) tc::tmem_dealloc(S.tslot, INFER_COLS);
}

}  // namespace mlp
}  // namespace hit
