// nonfinite.cuh -- count of NaN / Inf values in a float (or 16-bit) array, in two passes
// over a scratch array of per-block partial counts:
//   nonfinite_partial_kernel: block b counts values [b*NF_CHUNK, (b+1)*NF_CHUNK)
//                             and writes partials[b];
//   nonfinite_sum_kernel:     one block adds partials[0..nblocks) into
//                             partials[nblocks].
// Every slot used is written before it is read, so the scratch needs no
// clearing, and the result does not depend on the order blocks finish in.
#pragma once

#include <cstddef>
#include <cstdint>

namespace cgfd {
namespace nf {
// static: each translation unit that includes this gets its own copy

constexpr int NF_THREADS = 256;
constexpr int NF_ITEMS = 32;                         // values per thread
constexpr size_t NF_CHUNK = (size_t)NF_THREADS * NF_ITEMS;

static inline size_t nonfinite_blocks(size_t n) { return (n + NF_CHUNK - 1) / NF_CHUNK; }

static __device__ __forceinline__ unsigned long long nf_block_sum(unsigned long long v) {
  __shared__ unsigned long long warp_sums[NF_THREADS / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = v;
  __syncthreads();
  unsigned long long t = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < NF_THREADS / 32; ++w) t += warp_sums[w];
  return t;  // valid in thread 0
}

static __global__ void __launch_bounds__(NF_THREADS)
    nonfinite_partial_kernel(const float *__restrict__ v, size_t n,
                             unsigned long long *__restrict__ partials) {
  const size_t base = (size_t)blockIdx.x * NF_CHUNK;
  unsigned long long local = 0;
#pragma unroll 4
  for (int q = 0; q < NF_ITEMS; ++q) {
    const size_t o = base + (size_t)q * NF_THREADS + threadIdx.x;
    if (o < n && !isfinite(v[o])) ++local;
  }
  const unsigned long long t = nf_block_sum(local);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

// the same for 16-bit storage: a value is NaN or Inf when all its exponent
// bits (emask: 0x7C00 for IEEE half, 0x7F80 for bfloat16) are set
static __global__ void __launch_bounds__(NF_THREADS)
    nonfinite16_partial_kernel(const uint16_t *__restrict__ v, size_t n, uint16_t emask,
                               unsigned long long *__restrict__ partials) {
  const size_t base = (size_t)blockIdx.x * NF_CHUNK;
  unsigned long long local = 0;
#pragma unroll 4
  for (int q = 0; q < NF_ITEMS; ++q) {
    const size_t o = base + (size_t)q * NF_THREADS + threadIdx.x;
    if (o < n && (v[o] & emask) == emask) ++local;
  }
  const unsigned long long t = nf_block_sum(local);
  if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

static __global__ void __launch_bounds__(NF_THREADS)
    nonfinite_sum_kernel(unsigned long long *partials, int nblocks) {
  unsigned long long local = 0;
  for (int b = threadIdx.x; b < nblocks; b += NF_THREADS) local += partials[b];
  const unsigned long long t = nf_block_sum(local);
  if (threadIdx.x == 0) partials[nblocks] = t;
}

}  // namespace nf
}  // namespace cgfd
