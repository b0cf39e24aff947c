// Exclusive scan used by the order-preserving compactions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace umapb {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 16;                              // values per thread and pass
constexpr int64_t kScanPass = (int64_t)kScanThreads * kScanItems;  // 16 K values per pass
constexpr int kScanMaxBlocks = 64;

// Blocks and values per block of a scan of `count` values: ranges of at least one
// pass (16 K values), at most kScanMaxBlocks of them, each a multiple of 16 values so
// that every range starts on a 16-byte boundary when the array does.
inline void scan_shape(int64_t count, int* blocks, int64_t* span) {
  int64_t b = (count + kScanPass - 1) / kScanPass;
  if (b < 1) b = 1;
  if (b > kScanMaxBlocks) b = kScanMaxBlocks;
  int64_t s = (count + b - 1) / b;
  s = (s + 15) / 16 * 16;
  if (s < 16) s = 16;
  *blocks = (int)((count + s - 1) / s > 0 ? (count + s - 1) / s : 1);
  *span = s;
}

// Exclusive scan of `count` int32 values in place.  Block b owns [b span, (b + 1)
// span).  With more than one block, a first launch writes each block's range total
// to block_sums (it writes nothing to vals), and the scan launch starts block b from
// the sum of block_sums[0, b); the launch boundary orders the two, so no block reads a
// range another block is rewriting.  A block scans its range in passes of 16 K
// values: a thread scans its 16 consecutive values in registers, the block scans the
// thread sums (warp shuffles, then one warp over the 32 warp sums) and a running
// carry links the passes.  The last block writes the grand total to *total.
template <int kDummy = 0>
__global__ void __launch_bounds__(kScanThreads) scan_block_sums_kernel(const int32_t* __restrict__ vals,
                                                                       int64_t count, int64_t span,
                                                                       int64_t* __restrict__ block_sums) {
  __shared__ int64_t warp_sums[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t lo = (int64_t)blockIdx.x * span;
  const int64_t hi = lo + span < count ? lo + span : count;
  int64_t s = 0;
  if ((reinterpret_cast<uintptr_t>(vals) & 15) == 0) {
    const int64_t hi4 = lo + (hi - lo) / 4 * 4;  // lo is a multiple of 16
    for (int64_t i = lo + 4 * (int64_t)threadIdx.x; i < hi4; i += 4 * (int64_t)kScanThreads) {
      const int4 a = *reinterpret_cast<const int4*>(vals + i);
      s += (int64_t)a.x + a.y + a.z + a.w;
    }
    for (int64_t i = hi4 + threadIdx.x; i < hi; i += kScanThreads) s += vals[i];
  } else {
    for (int64_t i = lo + threadIdx.x; i < hi; i += kScanThreads) s += vals[i];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) warp_sums[warp] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int64_t t = 0;
    for (int w = 0; w < kScanThreads / 32; ++w) t += warp_sums[w];
    block_sums[blockIdx.x] = t;
  }
}

template <int kDummy = 0>
__global__ void __launch_bounds__(kScanThreads) scan_exclusive_kernel(int32_t* __restrict__ vals, int64_t count,
                                                                      int64_t span,
                                                                      const int64_t* __restrict__ block_sums,
                                                                      int64_t* __restrict__ total) {
  __shared__ int64_t warp_sums[32];
  __shared__ int64_t carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool aligned = (reinterpret_cast<uintptr_t>(vals) & 15) == 0;
  const int64_t lo = (int64_t)blockIdx.x * span;
  const int64_t hi = lo + span < count ? lo + span : count;
  if (threadIdx.x == 0) {  // the sum of vals[0, lo): the totals of the blocks before
    int64_t c = 0;
    for (int b = 0; b < (int)blockIdx.x; ++b) c += block_sums[b];
    carry = c;
  }
  __syncthreads();

  for (int64_t base = lo; base < hi; base += kScanPass) {
    const int64_t first = base + (int64_t)threadIdx.x * kScanItems;
    int32_t v[kScanItems];
    const bool full = aligned && first + kScanItems <= hi;
    if (full) {
#pragma unroll
      for (int q = 0; q < kScanItems / 4; ++q) {
        const int4 a = *reinterpret_cast<const int4*>(vals + first + 4 * q);
        v[4 * q] = a.x, v[4 * q + 1] = a.y, v[4 * q + 2] = a.z, v[4 * q + 3] = a.w;
      }
    } else {
#pragma unroll
      for (int u = 0; u < kScanItems; ++u) v[u] = first + u < hi ? vals[first + u] : 0;
    }
    int64_t sum = 0;
#pragma unroll
    for (int u = 0; u < kScanItems; ++u) sum += v[u];
    int64_t x = sum;  // inclusive scan of the thread sums within the warp
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int64_t s = warp_sums[lane];
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
    for (int u = 0; u < kScanItems; ++u) {  // exclusive prefix, in place
      const int32_t t = v[u];
      v[u] = (int32_t)run;
      run += t;
    }
    if (full) {
#pragma unroll
      for (int q = 0; q < kScanItems / 4; ++q)
        *reinterpret_cast<int4*>(vals + first + 4 * q) = make_int4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    } else {
#pragma unroll
      for (int u = 0; u < kScanItems; ++u)
        if (first + u < hi) vals[first + u] = v[u];
    }
    __syncthreads();
    if (threadIdx.x == kScanThreads - 1) carry = run;
    __syncthreads();
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *total = carry;
}

// Enqueue the scan of vals[0, count) (count >= 0) on `stream`; block_sums is caller
// scratch of kScanMaxBlocks int64 values (not read when one block covers count).
inline void scan_exclusive(int32_t* vals, int64_t count, int64_t* total, int64_t* block_sums, cudaStream_t stream) {
  int blocks;
  int64_t span;
  scan_shape(count, &blocks, &span);
  if (blocks > 1) {
    scan_block_sums_kernel<<<blocks, kScanThreads, 0, stream>>>(vals, count, span, block_sums);
    count_launches(1);  // the callers count the scan launch itself
  }
  scan_exclusive_kernel<<<blocks, kScanThreads, 0, stream>>>(vals, count, span, block_sums, total);
}

}  // namespace umapb
