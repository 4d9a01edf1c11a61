// Bulk asynchronous copies (TMA, cp.async.bulk) from global to shared memory
// completed on an mbarrier, for sm_90+ (here sm_100a). Non-multicast forms only.
//
// Rules these helpers assume: source and destination 16-byte aligned, sizes a
// multiple of 16 bytes. Waits are bounded: wait() gives up after `max_polls`
// polls and returns false, so a kernel can record an error instead of hanging.
#pragma once
#include <cstdint>

namespace cfg {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// arrive on the barrier and announce `bytes` of asynchronous transactions for this phase
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// global -> shared bulk copy completing `bytes` transactions on `bar`
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// shared -> global bulk copy (one bulk async-group per call): both addresses and `bytes`
// multiples of 16. The caller makes the block's shared-memory writes visible to the copy
// first (a block barrier, then proxy_fence_shared in the issuing thread) and waits with
// bulk_wait_read before that shared memory is written again or the block exits.
__device__ __forceinline__ void proxy_fence_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_addr(src)), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

// 2D tiled tensor copy global -> shared of the box at (x, y) of `tmap` (a CUtensorMap
// in global memory); out-of-range elements are zero-filled. x * element size must be
// a multiple of 16 bytes; the destination 128-byte aligned.
__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_addr(dst)),
      "l"(tmap), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}

// fetch a tensor map (a CUtensorMap in global memory that no kernel writes) into the
// descriptor cache ahead of the copies that name it
__device__ __forceinline__ void tmap_prefetch(const void* tmap) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(tmap) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded wait for phase `parity` of the barrier; false if it did not complete
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t max_polls = 1u << 22) {
  for (uint32_t k = 0; k < max_polls; k++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

}  // namespace cfg
