// Single-block exclusive scan used by the order-preserving compactions.
#pragma once

#include <stdint.h>

namespace umapb {

// Exclusive scan of `count` int32 values in place by ONE block of 1024 threads;
// writes the grand total to *total.
template <int kDummy = 0>
__global__ void scan_exclusive_kernel(int32_t* __restrict__ vals, int64_t count, int64_t* __restrict__ total) {
  __shared__ int64_t warp_sums[32];
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t base = 0; base < count; base += blockDim.x) {
    const int64_t idx = base + threadIdx.x;
    const int64_t v = idx < count ? vals[idx] : 0;
    int64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int64_t s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      warp_sums[lane] = s;
    }
    __syncthreads();
    const int64_t excl = carry + (warp > 0 ? warp_sums[warp - 1] : 0) + x - v;
    if (idx < count) vals[idx] = (int32_t)excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

}  // namespace umapb
