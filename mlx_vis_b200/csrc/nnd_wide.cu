// NNDescent for 32 < k <= 100 neighbours — the same iteration rules as the
// warp-per-row kernels of nndescent.cu (nndescent.py:103-378), one BLOCK per row:
//
//   candidates  [old row | first j_nn of the rows of its first mc_new neighbours
//               (NEW first on the converging path) | reverse row], the
//               reference's column order (up to 100 + 100 x 100 + 100 = 10,200)
//   dedup       first occurrence of every id kept: a shared-memory hash table
//               keyed by id holds the smallest column of the id (atomicMin)
//   distances   max(sq_i + sq_c - 2 x_i.x_c, 0) in the iteration's space, one warp
//               per candidate, the dot rounded to FP16 in the FP16 iterations; the
//               stored distance of an old neighbour unless the iteration recomputes
//   top-k       (distance bits << 32 | id) keys sorted by a block bitonic network;
//               self and duplicates sort last
//
// Shared memory per block: candidate ids and distances (8 B per column) + a
// 64-bit area of next_pow2(1.5 T) entries that holds the hash table and then the
// sort keys: 210 KB at k = 100, so one block per SM.
#include <cuda_fp16.h>
#include <stdint.h>

#include <mutex>

#include "common.cuh"
#include "nnd_wide.cuh"

namespace umapb {
namespace nnd_wide {

constexpr int kThreads = 512;
constexpr int kMaxK = 100;

__host__ __device__ inline int next_pow2(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

struct Shape {
  int T, tcap, H;  // columns, columns rounded to 32, 64-bit entries of the hash / sort area
  size_t smem;
};

inline Shape shape(int k, int mc, int j_nn, bool rev) {
  Shape s;
  s.T = k + mc * j_nn + (rev ? k : 0);
  s.tcap = (s.T + 31) / 32 * 32;
  s.H = next_pow2(s.tcap + s.tcap / 2);
  s.smem = (size_t)s.tcap * 8 + (size_t)s.H * 8 + 2 * (size_t)kMaxK * 4 + 64;
  return s;
}

template <class T>
__device__ __forceinline__ float to_f(T v);
template <>
__device__ __forceinline__ float to_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ float to_f<__half>(__half v) { return __half2float(v); }

// x_a . x_b over dd values of rows with pitch ld, by one warp (every lane gets it)
template <class T>
__device__ __forceinline__ float warp_dot(const T* __restrict__ X, int64_t a, int64_t b, int dd, int ld, int lane) {
  const T* xa = X + a * ld;
  const T* xb = X + b * ld;
  float acc = 0.f;
  for (int t = lane; t < dd; t += 32) acc = fmaf(to_f<T>(xa[t]), to_f<T>(xb[t]), acc);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  return acc;
}

__device__ __forceinline__ uint32_t hash_id(int32_t id) { return (uint32_t)id * 2654435761u; }

// ascending block bitonic sort of P (a power of two) 64-bit keys in shared memory
__device__ void block_sort(unsigned long long* key, int P) {
  for (int size = 2; size <= P; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = threadIdx.x; t < P / 2; t += blockDim.x) {
        const int lo = 2 * t - (t & (stride - 1));
        const int hi = lo + stride;
        const bool up = (lo & size) == 0;
        const unsigned long long a = key[lo], b = key[hi];
        if ((a > b) == up) {
          key[lo] = b;
          key[hi] = a;
        }
      }
      __syncthreads();
    }
  }
}

struct Args {
  const void* Xd;
  const float* sqd;
  int dd, ldx;
  const int32_t* idx_old;
  const float* dist_old;
  const uint8_t* flags_old;
  const int32_t* rev;
  int64_t n;
  int k, mc, j_nn;
  int converging, recompute_cur, half_round;
  int T, tcap, H;
  int32_t* idx_new;
  float* dist_new;
  uint8_t* flags_new;
  unsigned long long* changed;
  unsigned long long* evals;
};

template <class T>
__global__ void __launch_bounds__(kThreads) iter_kernel(Args a) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  unsigned long long* area = reinterpret_cast<unsigned long long*>(smem_raw);  // H entries
  int32_t* cid = reinterpret_cast<int32_t*>(area + a.H);
  float* cd = reinterpret_cast<float*>(cid + a.tcap);
  int32_t* src = reinterpret_cast<int32_t*>(cd + a.tcap);  // sources (kMaxK)
  __shared__ int s_flagged;
  __shared__ unsigned long long s_evals, s_changed;
  const int k = a.k;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const T* X = static_cast<const T*>(a.Xd);
  for (int64_t row = blockIdx.x; row < a.n; row += gridDim.x) {
    const int32_t* orow = a.idx_old + row * k;
    if (threadIdx.x == 0) {
      s_evals = 0;
      s_changed = 0;
      int f = 0;
      if (a.converging) {
        // NEW neighbours first, stable (nndescent.py:107-110)
        int m = 0;
        for (int p = 0; p < k; ++p)
          if (a.flags_old[row * k + p]) src[m++] = orow[p];
        f = m;
        for (int p = 0; p < k; ++p)
          if (!a.flags_old[row * k + p]) src[m++] = orow[p];
      } else {
        for (int p = 0; p < k; ++p) src[p] = orow[p];
        f = 1;
      }
      s_flagged = f;
    }
    __syncthreads();
    if (a.converging && s_flagged == 0) {  // no NEW neighbour: the row keeps its list
      for (int p = threadIdx.x; p < k; p += blockDim.x) {
        a.idx_new[row * k + p] = orow[p];
        a.dist_new[row * k + p] = a.dist_old[row * k + p];
        a.flags_new[row * k + p] = 0;
      }
      __syncthreads();
      continue;
    }
    // candidate columns in the reference's order
    const int nn_end = k + a.mc * a.j_nn;
    for (int t = threadIdx.x; t < a.T; t += blockDim.x) {
      int32_t id;
      if (t < k) {
        id = orow[t];
      } else if (t < nn_end) {
        const int q = t - k, p = q / a.j_nn, j = q - p * a.j_nn;
        id = a.idx_old[(int64_t)src[p] * k + j];
      } else {
        id = a.rev[row * k + (t - nn_end)];
      }
      cid[t] = id;
    }
    int32_t* hkey = reinterpret_cast<int32_t*>(area);
    int32_t* hval = hkey + a.H;
    for (int t = threadIdx.x; t < a.H; t += blockDim.x) {
      hkey[t] = -1;
      hval[t] = 0x7fffffff;
    }
    __syncthreads();
    // first occurrence of every id: the smallest column per id (H > T, so a free
    // slot always exists and every probe sequence ends)
    const uint32_t hm = (uint32_t)a.H - 1u;
    for (int t = threadIdx.x; t < a.T; t += blockDim.x) {
      const int32_t id = cid[t];
      uint32_t h = hash_id(id) & hm;
      for (;;) {
        const int32_t prev = atomicCAS(&hkey[h], -1, id);
        if (prev == -1 || prev == id) {
          atomicMin(&hval[h], t);
          break;
        }
        h = (h + 1) & hm;
      }
    }
    __syncthreads();
    // keep flags into cd: +inf for self / later duplicates, else to be computed
    for (int t = threadIdx.x; t < a.T; t += blockDim.x) {
      const int32_t id = cid[t];
      uint32_t h = hash_id(id) & hm;
      while (hkey[h] != id) h = (h + 1) & hm;
      const bool keep = hval[h] == t && id != (int32_t)row;
      cd[t] = keep ? -1.0f : INFINITY;
    }
    __syncthreads();
    // distances: stored ones for old neighbours unless recomputed, the rest by warps
    const float sq_i = a.sqd[row];
    unsigned long long my_evals = 0;
    for (int t = warp; t < a.T; t += nwarps) {
      if (cd[t] != -1.0f) continue;
      float d;
      if (t < k && !a.recompute_cur) {
        d = a.dist_old[row * k + t];
      } else {
        const int32_t c = cid[t];
        float dot = warp_dot<T>(X, row, c, a.dd, a.ldx, lane);
        if (a.half_round) dot = __half2float(__float2half_rn(dot));
        d = fmaxf(__fsub_rn(__fadd_rn(sq_i, a.sqd[c]), __fmul_rn(2.0f, dot)), 0.0f);
        ++my_evals;
      }
      if (lane == 0) cd[t] = d;
    }
    if (lane == 0 && my_evals) atomicAdd(&s_evals, my_evals);
    __syncthreads();
    // top-k of (distance, id): keys sorted ascending, padding and dropped columns last
    const int P = next_pow2(a.T);
    for (int t = threadIdx.x; t < P; t += blockDim.x) {
      unsigned long long key = ~0ull;
      if (t < a.T && cd[t] != INFINITY)
        key = ((unsigned long long)__float_as_uint(cd[t]) << 32) | (uint32_t)cid[t];
      area[t] = key;
    }
    __syncthreads();
    block_sort(area, P);
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
      const unsigned long long key = area[p];
      const int32_t id = (int32_t)(uint32_t)(key & 0xffffffffu);
      const float d = __uint_as_float((uint32_t)(key >> 32));
      a.idx_new[row * k + p] = id;
      a.dist_new[row * k + p] = d;
      const uint8_t ch = id != orow[p];
      a.flags_new[row * k + p] = ch;
      if (ch) atomicAdd(&s_changed, 1ull);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      if (s_changed) atomicAdd(a.changed, s_changed);
      if (a.evals && s_evals) atomicAdd(a.evals, s_evals);
    }
    __syncthreads();
  }
}

// Initial distances of the random graph (FP32) and, with sort_rows, each row
// ordered by (distance, id): one block per row.
__global__ void __launch_bounds__(256) gather_kernel(const float* __restrict__ X, const float* __restrict__ sq,
                                                     int64_t n, int dd, int32_t* __restrict__ idx,
                                                     float* __restrict__ dist, int k, int sort_rows) {
  __shared__ unsigned long long key[128];
  __shared__ float dv[kMaxK];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t row = blockIdx.x; row < n; row += gridDim.x) {
    for (int p = warp; p < k; p += blockDim.x >> 5) {
      const int32_t c = idx[row * k + p];
      const float dot = warp_dot<float>(X, row, c, dd, dd, lane);
      if (lane == 0) dv[p] = fmaxf(__fsub_rn(__fadd_rn(sq[row], sq[c]), __fmul_rn(2.0f, dot)), 0.0f);
    }
    __syncthreads();
    if (!sort_rows) {
      for (int p = threadIdx.x; p < k; p += blockDim.x) dist[row * k + p] = dv[p];
    } else {
      const int P = next_pow2(k);
      for (int t = threadIdx.x; t < P; t += blockDim.x)
        key[t] = t < k ? (((unsigned long long)__float_as_uint(dv[t]) << 32) | (uint32_t)idx[row * k + t]) : ~0ull;
      __syncthreads();
      block_sort(key, P);
      for (int p = threadIdx.x; p < k; p += blockDim.x) {
        idx[row * k + p] = (int32_t)(uint32_t)(key[p] & 0xffffffffu);
        dist[row * k + p] = __uint_as_float((uint32_t)(key[p] >> 32));
      }
    }
    __syncthreads();
  }
}

}  // namespace nnd_wide

int nnd_wide_max_k() { return nnd_wide::kMaxK; }

int nnd_gather_wide(const float* X, const float* sq, int64_t n, int dd, int32_t* idx, float* dist, int k,
                    int sort_rows, cudaStream_t stream) {
  UMAPB_REQUIRE(k > 32 && k <= nnd_wide::kMaxK, "nnd_gather: k must be <= %d", nnd_wide::kMaxK);
  const int64_t grid = n < (int64_t)num_sms() * 8 ? n : (int64_t)num_sms() * 8;
  nnd_wide::gather_kernel<<<(unsigned)grid, 256, 0, stream>>>(X, sq, n, dd, idx, dist, k, sort_rows);
  UMAPB_LAUNCH_CHECK("nnd_gather (k > 32) kernel");
  count_launches(1);
  return UMAPB_OK;
}

int nnd_iteration_wide(const void* Xd, const float* sqd, int dd, int ldx, int half, const int32_t* idx_old,
                       const float* dist_old, const uint8_t* flags_old, const int32_t* rev, int64_t n, int k,
                       int mc_new, int j_nn, int converging, int recompute_cur, int32_t* idx_new, float* dist_new,
                       uint8_t* flags_new, unsigned long long* changed, unsigned long long* evals,
                       cudaStream_t stream) {
  UMAPB_REQUIRE(k > 32 && k <= nnd_wide::kMaxK, "nnd_iteration: k must be <= %d", nnd_wide::kMaxK);
  const nnd_wide::Shape s = nnd_wide::shape(k, mc_new, j_nn, rev != nullptr);
  UMAPB_REQUIRE(s.smem <= 220 * 1024, "nnd_iteration: candidate list too long (%d columns)", s.T);
  static std::mutex mu;
  static bool attr[64] = {false};
  int dev = 0;
  UMAPB_CUDA_TRY(cudaGetDevice(&dev), "nnd_iteration: device");
  if (dev >= 0 && dev < 64) {
    std::lock_guard<std::mutex> lock(mu);
    if (!attr[dev]) {
      UMAPB_CUDA_TRY(cudaFuncSetAttribute(nnd_wide::iter_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          220 * 1024),
                     "nnd_iteration: smem attribute");
      UMAPB_CUDA_TRY(cudaFuncSetAttribute(nnd_wide::iter_kernel<__half>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024),
                     "nnd_iteration: smem attribute");
      attr[dev] = true;
    }
  }
  nnd_wide::Args a;
  a.Xd = Xd;
  a.sqd = sqd;
  a.dd = dd;
  a.ldx = ldx;
  a.idx_old = idx_old;
  a.dist_old = dist_old;
  a.flags_old = flags_old;
  a.rev = rev;
  a.n = n;
  a.k = k;
  a.mc = mc_new;
  a.j_nn = j_nn;
  a.converging = converging;
  a.recompute_cur = recompute_cur;
  a.half_round = half;
  a.T = s.T;
  a.tcap = s.tcap;
  a.H = s.H;
  a.idx_new = idx_new;
  a.dist_new = dist_new;
  a.flags_new = flags_new;
  a.changed = changed;
  a.evals = evals;
  int per_sm = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, half ? (const void*)nnd_wide::iter_kernel<__half>
                                                                   : (const void*)nnd_wide::iter_kernel<float>,
                                                    nnd_wide::kThreads, s.smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  cudaGetLastError();
  int64_t grid = (int64_t)num_sms() * per_sm;
  if (grid > n) grid = n;
  if (half)
    nnd_wide::iter_kernel<__half><<<(unsigned)grid, nnd_wide::kThreads, s.smem, stream>>>(a);
  else
    nnd_wide::iter_kernel<float><<<(unsigned)grid, nnd_wide::kThreads, s.smem, stream>>>(a);
  UMAPB_LAUNCH_CHECK("nnd_iteration (k > 32) kernel");
  count_launches(1);
  return UMAPB_OK;
}

}  // namespace umapb
