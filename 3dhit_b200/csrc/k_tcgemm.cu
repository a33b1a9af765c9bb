// BF16 GEMM on the fifth-generation tensor cores (tcgen05, sm_100a):
//   C[M][N] (float32, row-major) = A[M][K] (bf16, row-major) * B[N][K]^T (bf16, row-major)
// One CTA of 128 threads per 128-row tile of C; N in {16, 32, 64, 128};
// K a multiple of 16.  The K dimension is walked in chunks of 64: the chunk's
// A (128 x 64) and B (N x 64) tiles are copied to shared memory in the K-major
// core-matrix layout (tc_common.cuh), one thread issues the chunk's four
// K = 16 MMAs into the F32 accumulator in TMEM and commits them to an
// mbarrier; the accumulator is read back with tcgen05.ld (thread t owns row t).
//
// Every wait is bounded: if an MMA never completes the CTA raises *err,
// frees its TMEM and returns.
#include <cuda_bf16.h>

#include "kernels.h"
#include "tc_common.cuh"

namespace hit {

namespace {
constexpr int TC_KC = 64;        // K chunk
constexpr int TC_WAIT = 1 << 22;  // mbarrier poll limit
}  // namespace

// Split K: CTA (x, y) sums K columns [y*kslice, min((y+1)*kslice, K)) into
// C + y*cstride (one partial per split; kslice a multiple of 16).
template <int N>
__global__ void __launch_bounds__(128) k_tcgemm(const __nv_bfloat16* __restrict__ A, int lda,
                                                const __nv_bfloat16* __restrict__ B, int ldb, float* __restrict__ C,
                                                int ldc, int M, int K, int kslice, long long cstride, int* err) {
  static_assert(N == 16 || N == 32 || N == 64 || N == 128, "N");
  constexpr int NCOL = N < 32 ? 32 : N;  // TMEM columns (power of two >= 32)
  __shared__ __align__(1024) unsigned char sA[128 * TC_KC * 2];
  __shared__ __align__(1024) unsigned char sB[N * TC_KC * 2];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m0 = blockIdx.x * 128;
  const uint32_t mb = tc::smem_u32(&mbar);
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(&tslot), NCOL);
  if (tid == 0) tc::mbar_init(mb, 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tslot;
  const uint32_t idesc = tc::idesc_bf16(128, N);
  bool ok = true;
  uint32_t phase = 0;
  const int kbeg = blockIdx.y * kslice, kend = min(K, kbeg + kslice);
  C += blockIdx.y * cstride;
  if (kbeg >= kend) {  // empty split: a zero partial
    for (int e = tid; e < 128 * N; e += 128) {
      const int r = m0 + e / N;
      if (r < M) C[(long long)r * ldc + e % N] = 0.f;
    }
  }
  for (int k0 = kbeg; k0 < kend && ok; k0 += TC_KC) {
    const int kc = min(TC_KC, kend - k0);  // multiple of 16
    // A chunk: 128 rows x kc, 8 bf16 (16 bytes) per copy, zero rows past M
    for (int e = tid; e < 128 * (kc / 8); e += 128) {
      const int r = e / (kc / 8), c8 = e % (kc / 8);
      uint4 v = make_uint4(0, 0, 0, 0);
      if (m0 + r < M) v = *reinterpret_cast<const uint4*>(A + (long long)(m0 + r) * lda + k0 + c8 * 8);
      *reinterpret_cast<uint4*>(sA + tc::kmajor_off(r, c8 * 8, TC_KC)) = v;
    }
    for (int e = tid; e < N * (kc / 8); e += 128) {
      const int r = e / (kc / 8), c8 = e % (kc / 8);
      *reinterpret_cast<uint4*>(sB + tc::kmajor_off(r, c8 * 8, TC_KC)) =
          *reinterpret_cast<const uint4*>(B + (long long)r * ldb + k0 + c8 * 8);
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
      const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
      for (int s = 0; s < kc / 16; ++s)
        tc::mma_bf16(tmem, tc::smem_desc(a0 + 256 * s, 128, TC_KC * 16), tc::smem_desc(b0 + 256 * s, 128, TC_KC * 16),
                     idesc, k0 > kbeg || s > 0);
      tc::commit(mb);
    }
    // the tiles may be overwritten once the MMAs are done; the verdict is block-uniform
    ok = __syncthreads_and(tc::mbar_wait(mb, phase, TC_WAIT)) != 0;
    phase ^= 1;
    tc::fence_after_sync();
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
  } else if (kbeg < kend) {
    const int row = m0 + tid;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int c0 = 0; c0 < N; c0 += 16) {
      float v[16];
      tc::tmem_ld16(lane_addr + c0, v);
      if (row < M) {
#pragma unroll
        for (int i = 0; i < 16; ++i) C[(long long)row * ldc + c0 + i] = v[i];
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tmem, NCOL);
}

// sum of `splits` partials [splits][M][N] into C[M][N] (fixed order)
__global__ void k_sum_splits(const float* __restrict__ part, float* __restrict__ C, long long n, int splits) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int y = 0; y < splits; ++y) s += part[y * n + i];
    C[i] = s;
  }
}

cudaError_t launch_tcgemm(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, float* C, int ldc, int M,
                          int N, int K, int* err, cudaStream_t st, int splits, float* work) {
  if (M < 1 || K < 16 || K % 16 || lda % 8 || ldb % 8 || splits < 1) return cudaErrorInvalidValue;
  // K slices of whole 16-column steps
  const int steps = K / 16, per = (steps + splits - 1) / splits, kslice = per * 16;
  float* out = splits > 1 ? work : C;
  const long long cstride = (long long)M * N;
  const dim3 grid((M + 127) / 128, splits);
  const int ldo = splits > 1 ? N : ldc;
  switch (N) {
    case 16: k_tcgemm<16><<<grid, 128, 0, st>>>(A, lda, B, ldb, out, ldo, M, K, kslice, cstride, err); break;
    case 32: k_tcgemm<32><<<grid, 128, 0, st>>>(A, lda, B, ldb, out, ldo, M, K, kslice, cstride, err); break;
    case 64: k_tcgemm<64><<<grid, 128, 0, st>>>(A, lda, B, ldb, out, ldo, M, K, kslice, cstride, err); break;
    case 128: k_tcgemm<128><<<grid, 128, 0, st>>>(A, lda, B, ldb, out, ldo, M, K, kslice, cstride, err); break;
    default: return cudaErrorInvalidValue;
  }
  if (splits > 1) {
    if (ldc != N) return cudaErrorInvalidValue;  // the partials are dense
    k_sum_splits<<<(int)std::min<long long>((cstride + 255) / 256, 4 * 148), 256, 0, st>>>(work, C, cstride, splits);
  }
  return cudaGetLastError();
}

}  // namespace hit
