// Single-block exclusive scan used by the order-preserving compactions.
#pragma once

#include <stdint.h>

namespace umapb {

// Exclusive scan of `count` int32 values in place by ONE block of 1024 threads;
// writes the grand total to *total.  Each pass covers 1024 x 16 values (one pass
// for up to 16 K values, five for 70 K): a thread scans its 16 consecutive values
// in registers (four 16-byte loads), the block scans the thread sums (warp
// shuffles, then one warp over the 32 warp sums) and a running carry links the
// passes.
template <int kDummy = 0>
__global__ void __launch_bounds__(1024) scan_exclusive_kernel(int32_t* __restrict__ vals, int64_t count,
                                                              int64_t* __restrict__ total) {
  constexpr int kItems = 16;
  __shared__ int64_t warp_sums[32];
  __shared__ int64_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t span = (int64_t)blockDim.x * kItems;
  const bool aligned = (reinterpret_cast<uintptr_t>(vals) & 15) == 0;
  for (int64_t base = 0; base < count; base += span) {
    const int64_t first = base + (int64_t)threadIdx.x * kItems;
    int32_t v[kItems];
    const bool full = aligned && first + kItems <= count;
    if (full) {
#pragma unroll
      for (int q = 0; q < kItems / 4; ++q) {
        const int4 a = *reinterpret_cast<const int4*>(vals + first + 4 * q);
        v[4 * q] = a.x, v[4 * q + 1] = a.y, v[4 * q + 2] = a.z, v[4 * q + 3] = a.w;
      }
    } else {
#pragma unroll
      for (int u = 0; u < kItems; ++u) v[u] = first + u < count ? vals[first + u] : 0;
    }
    int64_t sum = 0;
#pragma unroll
    for (int u = 0; u < kItems; ++u) sum += v[u];
    int64_t x = sum;  // inclusive scan of the thread sums within the warp
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
    int64_t run = carry + (warp > 0 ? warp_sums[warp - 1] : 0) + x - sum;
#pragma unroll
    for (int u = 0; u < kItems; ++u) {  // exclusive prefix, in place
      const int32_t t = v[u];
      v[u] = (int32_t)run;
      run += t;
    }
    if (full) {
#pragma unroll
      for (int q = 0; q < kItems / 4; ++q)
        *reinterpret_cast<int4*>(vals + first + 4 * q) = make_int4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    } else {
#pragma unroll
      for (int u = 0; u < kItems; ++u)
        if (first + u < count) vals[first + u] = v[u];
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = run;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

}  // namespace umapb
