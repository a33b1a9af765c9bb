// Fifth-generation tensor-core (tcgen05) building blocks for sm_100a: TMEM
// allocation, shared-memory and instruction descriptors for BF16 x BF16 -> F32
// MMAs, the single-thread MMA issue with completion through an mbarrier, and
// TMEM loads.
//
// Operand layout in shared memory ("K-major, no swizzle"): a tile of R rows
// (M or N) by KC columns (K, bf16) is stored as 8 x 8 core matrices of 128
// contiguous bytes (8 rows of 16 bytes); element (r, k) lives at byte
//   (r / 8) * SBO + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,  SBO = KC * 16,
// so the leading-dimension byte offset (next 8-column group) is 128 and the
// stride byte offset (next 8-row group) is KC * 16.  One MMA consumes K = 16,
// i.e. two core-matrix columns; its descriptor starts 256 bytes further per
// K step.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace hit {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (r, k) in a K-major no-swizzle tile with KC columns.
__host__ __device__ constexpr uint32_t kmajor_off(int r, int k, int KC) {
  return (uint32_t)((r >> 3) * (KC * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor (version 1, no swizzle, base offset 0).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: BF16 A and B, F32 accumulator, both
// operands K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D(tmem) (+)= A(smem desc) * B(smem desc); issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"((uint32_t)accumulate));
}

// Arrive on the mbarrier once every MMA this thread issued has completed.
__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// Bounded wait for the phase with parity `parity` to complete; false when the
// limit is reached first.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, int limit) {
  for (int i = 0; i < limit; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// Generic-proxy shared-memory writes become visible to the tensor cores.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM allocation (one full warp; ncols a power of two >= 32): the base
// address is written to shared memory at `slot`.
__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive 32-bit columns of this thread's TMEM lane (warp w reads lanes
// 32w .. 32w+31; taddr carries the lane in its upper 16 bits).  The load and
// its completion wait are one asm statement, so no instruction can read the
// destination registers before they are filled.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 8 consecutive columns, as tmem_ld16.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// 16 consecutive 32-bit columns of this thread's TMEM lane from registers
// (asynchronous: tmem_wait_st before the columns are read back).
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
          taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
      "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
      "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])),
      "r"(__float_as_uint(v[11])), "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])),
      "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15]))
      : "memory");
}
// Two consecutive columns (one complex value) at each of taddr + k*d, k = 0..2.
__device__ __forceinline__ void tmem_st2x3(uint32_t taddr, uint32_t d, const float (&v)[6]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%3,%4};\n\t"
      "tcgen05.st.sync.aligned.32x32b.x2.b32 [%1], {%5,%6};\n\t"
      "tcgen05.st.sync.aligned.32x32b.x2.b32 [%2], {%7,%8};" ::"r"(taddr),
      "r"(taddr + d), "r"(taddr + 2 * d), "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])),
      "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5]))
      : "memory");
}
// The loads of tmem_st2x3's pattern at two bases (taddr, taddr + e), with
// their completion wait in the same asm statement.
__device__ __forceinline__ void tmem_ld2x3x2(uint32_t taddr, uint32_t d, uint32_t e, float (&v)[12]) {
  uint32_t r[12];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0,%1}, [%12];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%2,%3}, [%13];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%4,%5}, [%14];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%6,%7}, [%15];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%8,%9}, [%16];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%10,%11}, [%17];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11])
      : "r"(taddr), "r"(taddr + d), "r"(taddr + 2 * d), "r"(taddr + e), "r"(taddr + e + d), "r"(taddr + e + 2 * d)
      : "memory");
#pragma unroll
  for (int i = 0; i < 12; ++i) v[i] = __uint_as_float(r[i]);
}
// Wait until this thread's earlier tcgen05.st have completed.
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

}  // namespace tc
}  // namespace hit
