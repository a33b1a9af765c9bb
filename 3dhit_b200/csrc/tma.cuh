// Tensor-memory-accelerator (TMA) tile loads for the column transforms: a
// 4-D tiled tensor map over a (component, outer, row, z) array, loads issued by
// one thread with completion counted in bytes on an mbarrier, and a bounded
// wait.  Only loads (no stores, no multicast); the z coordinate of every load
// is a multiple of 8 elements (64 bytes), the tensor map's strides are
// multiples of 16 bytes and its box is 64 bytes wide.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace hit {
namespace tma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// This thread's arrival, announcing `bytes` of TMA transactions for the phase.
__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

// Bounded wait for the phase of parity `parity`; false when the limit is hit.
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

// Box at coordinates (x, y, z, w) of `map` into shared memory at dst (128-byte
// aligned), completing on mbar.
__device__ __forceinline__ void load4(void* dst, const CUtensorMap* map, int x, int y, int z, int w, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(mbar)
      : "memory");
}

// Contiguous bytes (16-byte aligned addresses, a multiple of 16 bytes) from
// global into shared memory, completing on mbar.
__device__ __forceinline__ void load_bytes(void* dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(mbar)
      : "memory");
}

// Generic-proxy shared-memory writes ordered before later async-proxy (TMA)
// accesses.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

}  // namespace tma
}  // namespace hit
