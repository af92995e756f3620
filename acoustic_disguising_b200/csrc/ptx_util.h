// ptx_util.h -- mbarrier and bulk-copy wrappers shared by the kernels.
#pragma once
#include <stdint.h>

namespace adf {

// Upper bound on mbarrier polls before a wait reports failure.
constexpr uint32_t kWaitLimit = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t a, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t a, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t a) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t a, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(a), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after kWaitLimit polls so that a logic error
// surfaces as an error code instead of a hung GPU.  try_wait itself suspends
// the thread for a bounded, hardware-chosen interval, so the loop does not
// spin hot and wakes as soon as the phase completes.
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity,
                                          uint32_t limit = kWaitLimit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(a, parity)) return true;
  return false;
}
// One-dimensional bulk copy global -> this CTA's shared memory, completing on
// an mbarrier.  dst and src 16-B aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes,
                                          uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(dst), "l"((uint64_t)src), "r"(bytes), "r"(mbar)
      : "memory");
}
// Four-dimensional tiled TMA load of one box global -> this CTA's shared
// memory, completing on an mbarrier.  `map` is a CUtensorMap in global
// memory (64-B aligned); the innermost coordinate x times the element size
// must be a multiple of 16 bytes.  No multicast.
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const void* map, int x, int y, int z,
                                            int c, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(c), "r"(mbar)
      : "memory");
}
// The same for a three-dimensional map.
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const void* map, int x, int y, int z,
                                            uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(z), "r"(mbar)
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

}  // namespace adf
