// tdf_bulk.cuh -- asynchronous bulk copies global -> shared memory for sm_100a:
// tiled TMA loads (cp.async.bulk.tensor, no multicast) completing on
// mbarrier transaction counts, and bounded waits on those barriers.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace tdf {

// or-ed into a kernel's error word when a bounded wait on a copy gave up
constexpr unsigned ERR_STAGE_TIMEOUT = 2u;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
     return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
     asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// makes barrier initialisation visible to the asynchronous (TMA) proxy
__device__ __forceinline__ void mbar_fence_init() {
     asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// one arrival that also announces `bytes` of transactions still to come
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
     asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                  : "memory");
}

// Waits for the phase of `parity` to complete, giving up after `limit`
// probes (each probe may suspend the thread for a hardware-defined time).
// Returns false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int limit = 1 << 20) {
     const uint32_t a = smem_addr(bar);
     for (int it = 0; it < limit; it++) {
          uint32_t done;
          asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
              "selp.u32 %0, 1, 0, p;\n\t}"
              : "=r"(done)
              : "r"(a), "r"(parity)
              : "memory");
          if (done) return true;
     }
     return false;
}

// 1-D bulk copy of `bytes` (a multiple of 16; both addresses 16-byte
// aligned) from global to shared memory, completing on `bar` (no multicast).
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
     asm volatile(
         "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
             smem_addr(dst)),
         "l"((uint64_t)src), "r"(bytes), "r"(smem_addr(bar))
         : "memory");
}

// Tiled 3-D TMA load of one box into shared memory (no multicast); x as
// for tma_load_4d.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
     asm volatile(
         "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
         " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
         "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
         : "memory");
}

// Tiled 4-D TMA load of one box into shared memory (no multicast).  The
// innermost coordinate x times the element size must be a multiple of 16
// bytes; callers only pass x that are multiples of 8 elements of 4 bytes.
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int x, int y, int z, int w,
                                            uint64_t *bar) {
     asm volatile(
         "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
         " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
         "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_addr(bar))
         : "memory");
}

// Per-thread asynchronous copies global -> shared memory of 16 or 8 bytes
// (both addresses aligned to the size), waited for with cp_async_wait_all();
// a thread's copies are all in flight at once and hold no registers.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
     asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"((uint64_t)src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
     asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"((uint64_t)src) : "memory");
}
// the calling thread's copies have landed (other threads' need a barrier)
__device__ __forceinline__ void cp_async_wait_all() {
     asm volatile("cp.async.wait_all;" ::: "memory");
}

}  // namespace tdf
