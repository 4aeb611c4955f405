// Tensor Memory Accelerator copies between global and shared memory, and the
// shared-memory barriers that track them (sm_100a PTX). Every wait is bounded:
// a copy that has not landed after kTmaWaitNs sets the caller's error word and
// the kernel returns without using the tile.
#pragma once

#include <cuda.h>  // CUtensorMap
#include <stdint.h>

namespace bz {

constexpr unsigned long long kTmaWaitNs = 100000000ull;  // 100 ms per copy

#if defined(__CUDACC__)
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ unsigned long long tma_clock_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// One thread: a barrier expecting one arrival (the issuing thread's), made
// visible to the async proxy before any copy signals it.
__device__ __forceinline__ void mbar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// The issuing thread's arrival, announcing `bytes` of copies to come.
__device__ __forceinline__ void mbar_expect(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// Waits until phase `parity` of the barrier has completed; false after kTmaWaitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_addr(bar);
  const unsigned long long t0 = tma_clock_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (tma_clock_ns() - t0 > kTmaWaitNs) return false;
  }
}

// Contiguous copy global -> shared (16-byte aligned addresses, size a
// multiple of 16), completing on `bar`.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Contiguous copy shared -> global, in the thread's current bulk group.
__device__ __forceinline__ void bulk_store(void *dst, const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
               "r"(smem_addr(src)), "r"(bytes)
               : "memory");
}

// Box of a 3-D tensor map at coordinates (x, y, z) -> shared, completing on `bar`.
__device__ __forceinline__ void tensor_load_3d(void *dst, const CUtensorMap *map, int x, int y,
                                               int z, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

// shared -> box of a 3-D tensor map at (x, y, z), in the thread's current bulk group.
__device__ __forceinline__ void tensor_store_3d(const CUtensorMap *map, int x, int y, int z,
                                                const void *src) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::
                   "l"(map),
               "r"(x), "r"(y), "r"(z), "r"(smem_addr(src))
               : "memory");
}

// Closes the thread's bulk group and waits until its copies have read their
// shared-memory source (the tile may then be reused or the block may exit).
__device__ __forceinline__ void bulk_store_drain() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// Every thread that wrote shared memory the async proxy will read, before
// the block barrier that precedes the store.
__device__ __forceinline__ void fence_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
#endif

}  // namespace bz
