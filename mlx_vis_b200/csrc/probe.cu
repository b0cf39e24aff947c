// Access-rate probes: the measured ceilings of the two gather-bound steps of the
// pipeline, timed by the caller around one launch (bench.py reports the layout epoch
// and the NNDescent join against them).
//
//   umapb_probe_random_access: each thread makes `per_thread` rounds of one random
//     row read of `dim` floats from `table` (n rows) and, every `red_every` rounds,
//     one random float atomic add of `dim` values into `dtable`: the access mix of a
//     layout epoch (about 7 gathers to 2 atomics per edge), rows drawn by a hash.
//   umapb_probe_row_gather: one warp per entry of `ids` reads the whole row
//     `row_bytes` long (16-byte loads, lanes striding the row) from `table`, as the
//     NNDescent join reads its candidate rows.
#include "common.cuh"

namespace umapb {
namespace probe {

__device__ __forceinline__ uint32_t mix32(uint32_t x) {  // a 32-bit integer hash (xorshift-multiply)
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

template <int DIM>
__global__ void random_access_kernel(const float* __restrict__ table, float* __restrict__ dtable, int n,
                                     int per_thread, int red_every, float* __restrict__ sink) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t s = mix32(tid * 2654435761u + 12345u);
  float acc = 0.f;
  for (int r = 0; r < per_thread; ++r) {
    s = mix32(s + (uint32_t)r);
    const int row = (int)(((uint64_t)s * (uint64_t)n) >> 32);
    const float* p = table + (int64_t)row * DIM;
    if constexpr (DIM == 2) {
      const float2 v = __ldg(reinterpret_cast<const float2*>(p));
      acc += v.x + v.y;
    } else {
#pragma unroll
      for (int c = 0; c < DIM; ++c) acc += __ldg(p + c);
    }
    if (red_every > 0 && r % red_every == 0) {
      const int t = (int)(((uint64_t)mix32(s ^ 0x9e3779b9u) * (uint64_t)n) >> 32);
      const float v = 1e-30f * acc;  // vector atomics, as the layout's moves
      if constexpr (DIM == 2) {
        atomicAdd(reinterpret_cast<float2*>(dtable) + t, make_float2(v, v));
      } else if constexpr (DIM == 4) {
        atomicAdd(reinterpret_cast<float4*>(dtable) + t, make_float4(v, v, v, v));
      } else {
        atomicAdd(dtable + t, v);
      }
    }
  }
  if (acc == 1.234567f) sink[0] = acc;  // keeps the loads; practically never stores
}

__global__ void row_gather_kernel(const int4* __restrict__ table, int64_t rows, int row_int4,
                                  const int32_t* __restrict__ ids, int64_t count, int4* __restrict__ sink) {
  const int lane = threadIdx.x & 31;
  int4 acc = make_int4(0, 0, 0, 0);
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < count; w += warps) {
    const int64_t id = ids[w];
    if (id < 0 || id >= rows) continue;  // out-of-range entries are skipped
    const int4* r = table + id * row_int4;
    for (int q = lane; q < row_int4; q += 32) {
      const int4 v = __ldcg(r + q);
      acc.x ^= v.x;
      acc.y ^= v.y;
      acc.z ^= v.z;
      acc.w ^= v.w;
    }
  }
  if (acc.x == 0x13579bdf && acc.y == 0x2468ace0) sink[0] = acc;
}

}  // namespace probe
}  // namespace umapb

using namespace umapb;

extern "C" int umapb_probe_random_access(const float* table, float* dtable, int64_t n, int32_t dim, int64_t threads,
                                         int32_t per_thread, int32_t red_every, float* sink,
                                         umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(table && sink && (dtable || red_every <= 0), "probe_random_access: null argument");
  UMAPB_REQUIRE(n >= 1 && n < ((int64_t)1 << 31) && (dim == 1 || dim == 2 || dim == 4),
                "probe_random_access: need 1 <= n < 2^31 and dim 1, 2 or 4");
  UMAPB_REQUIRE(threads >= 256 && threads % 256 == 0 && threads / 256 < ((int64_t)1 << 31) && per_thread >= 1,
                "probe_random_access: threads a positive multiple of 256, per_thread >= 1");
  const unsigned blocks = (unsigned)(threads / 256);
  switch (dim) {
    case 1: probe::random_access_kernel<1><<<blocks, 256, 0, stream>>>(table, dtable, (int)n, per_thread, red_every, sink); break;
    case 2: probe::random_access_kernel<2><<<blocks, 256, 0, stream>>>(table, dtable, (int)n, per_thread, red_every, sink); break;
    default: probe::random_access_kernel<4><<<blocks, 256, 0, stream>>>(table, dtable, (int)n, per_thread, red_every, sink); break;
  }
  UMAPB_LAUNCH_CHECK("probe_random_access kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_probe_row_gather(const void* table, int64_t rows, int32_t row_bytes, const int32_t* ids,
                                      int64_t count, void* sink, umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(table && ids && sink && rows >= 1 && count >= 0, "probe_row_gather: bad arguments");
  UMAPB_REQUIRE(row_bytes >= 16 && row_bytes % 16 == 0 && (reinterpret_cast<uintptr_t>(table) & 15) == 0,
                "probe_row_gather: rows must be 16-byte multiples on a 16-byte aligned table");
  if (count == 0) return UMAPB_OK;
  const int64_t want = ceil_div(count, 8);  // 8 warps per block
  const int64_t cap = (int64_t)num_sms() * 8;
  probe::row_gather_kernel<<<(unsigned)(want < cap ? want : cap), 256, 0, stream>>>(
      static_cast<const int4*>(table), rows, row_bytes / 16, ids, count, static_cast<int4*>(sink));
  UMAPB_LAUNCH_CHECK("probe_row_gather kernel");
  count_launches(1);
  return UMAPB_OK;
}
