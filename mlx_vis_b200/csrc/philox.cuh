// Counter-based random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11).  Stateless: the
// output is a pure function of (counter, key), so any thread can draw any
// element of a stream independently.
#pragma once

#include <stdint.h>

namespace umapb {

struct U4 {
  uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// Uniform integer in [0, n) from 32 random bits (multiply-high; bias < n / 2^32).
__device__ __forceinline__ int to_range(uint32_t r, uint32_t n) {
  return (int)(((uint64_t)r * (uint64_t)n) >> 32);
}

// Uniform float in (0, 1] from 32 random bits.
__device__ __forceinline__ float to_unit(uint32_t r) {
  return ((float)(r >> 8) + 1.0f) * (1.0f / 16777216.0f);
}

}  // namespace umapb
