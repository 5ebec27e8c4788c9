// r3d_async.cuh -- the asynchronous copy engine from device code: mbarriers,
// bulk copies (cp.async.bulk) and tiled tensor copies (cp.async.bulk.tensor)
// between global and shared memory.  No multicast forms.
#pragma once

#include <stdint.h>

namespace r3d {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// 16-byte asynchronous copies global -> shared through L2 (cp.async); they
// complete by groups: commit after a set of copies, then wait for all
// committed groups.  A hardware wait on copies already issued (no spin).
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)),
               "l"(__cvta_generic_to_global(src))
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}
// Bounded wait for phase `parity` of `bar`; false when the limit ran out.
// polls <= 0: the default, 2^22 polls of try_wait (far beyond any copy's
// latency).  polls > 0 (the test hook of the error path): that many
// non-blocking test_wait polls, which a copy issued just before the wait
// does not satisfy.
constexpr int kWaitPolls = 1 << 22;
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int polls = 0) {
  if (polls > 0) {
    for (int it = 0; it < polls; ++it) {
      uint32_t done;
      asm volatile(
          "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
          " selp.u32 %0, 1, 0, p;\n}"
          : "=r"(done)
          : "r"(smem_u32(bar)), "r"(parity)
          : "memory");
      if (done) return true;
    }
    return false;
  }
  for (int it = 0; it < kWaitPolls; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}


// Tiled tensor copies through a tensor map (CUtensorMap, 128 bytes, 64-byte
// aligned, in global memory); coordinates innermost first, in elements.
__device__ __forceinline__ void tma_load_4d(void *dst, const void *tmap, int c0, int c1, int c2,
                                            int c3, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_store_4d(const void *tmap, int c0, int c1, int c2, int c3,
                                             const void *src) {
  asm volatile(
      "cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::
          "l"(tmap),
      "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(src))
      : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// wait until this thread's committed bulk stores have finished reading
// shared memory (the buffer may be overwritten)
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// wait until this thread's committed bulk stores have completed
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}
// generic-proxy writes to shared memory become visible to the async proxy
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace r3d
