// ptx_util.cuh -- inline-PTX helpers of the TMA-fed stage kernels (sm_100a):
// mbarriers with bounded waits, 4-D tensor copies into shared memory and
// 4-D tensor prefetches into L2.  No multicast form is used anywhere.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace cgfd {
namespace ptx {

// every mbarrier wait gives up after this much %globaltimer time (microseconds)
constexpr unsigned WAIT_US = 2000000u;

__device__ __forceinline__ uint32_t su32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t n) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long gtime() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// bounded wait on the phase of the given parity; false after limit_us of
// %globaltimer time
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity,
                                          unsigned limit_us = WAIT_US) {
  if (mbar_try_wait(b, parity)) return true;
  const unsigned long long t0 = gtime(), lim = 1000ull * limit_us;
  while (!mbar_try_wait(b, parity))
    if (gtime() - t0 > lim) return false;
  return true;
}
// box at (x, y, z, c) of a 4-D tensor map into shared memory, completing on
// the mbarrier; x times the element size must be a multiple of 16 bytes (the callers' tiles
// start on 16-byte boundaries by construction)
__device__ __forceinline__ void tma_load(void *dst, const CUtensorMap *map, int x, int y, int z,
                                         int c, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(su32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(c), "r"(su32(bar))
      : "memory");
}
// the same box into L2 only (a hint: nothing waits for it)
__device__ __forceinline__ void tma_prefetch(const CUtensorMap *map, int x, int y, int z, int c) {
  asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];" ::"l"(map),
               "r"(x), "r"(y), "r"(z), "r"(c)
               : "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

}  // namespace ptx
}  // namespace cgfd
