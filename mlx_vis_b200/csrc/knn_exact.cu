// Exact brute-force kNN for long candidate lists (k + extra > 128) — the chunked
// loop of mlx_vis/_knn.py:47-88 for any k up to 4096:
//
//   D = max(|x_i|^2 + |x_j|^2 - 2 x_i.x_j, 0), self excluded, the k smallest per row
//   by (distance, index), sqrt unless squared.
//
// X is split once into three BF16 parts (umapb_split3); each block of R query rows
// gets its dot products against all n rows from the split-precision tcgen05 GEMM
// (FP32-level error, umapb_gemm_split3) into an (R, n) FP32 tile, then one CTA per
// query row selects L = k + extra candidates by that formula: a 4-pass 8-bit radix
// select finds the L-th key (distance bits; the row's keys sit in shared memory when
// they fit), the keys below it and the first of the keys equal to it (lowest indices)
// are gathered; each candidate's distance is then recomputed exactly in FP32 as
// sum (x_i - x_j)^2 (one warp per candidate; the expansion cancels for near
// duplicates, 1e-4 of |x|^2 here), a bitonic sort of (distance bits, index) orders
// them and the first k are written -- the rerank of the short-list path.
#include <cuda_bf16.h>
#include <math.h>

#include <mutex>

#include "common.cuh"
#include "knn_exact.cuh"

extern "C" int umapb_split3(const float* S, int64_t rows, int64_t cols, int64_t lds, const float* mu,
                            int32_t transpose, int32_t kp, void* out, umapb_stream_t stream);
extern "C" int umapb_gemm_split3(const void* A3, const void* B3, int32_t M, int32_t N, int32_t kp, int32_t ksplit,
                                 float* C, int32_t ldc, int32_t* status, umapb_stream_t stream);
extern "C" int umapb_nnd_sqnorms(const void* X, int64_t n, int32_t dd, int32_t half, float* sq,
                                 umapb_stream_t stream);

namespace umapb {
namespace knnx {

constexpr int kThreads = 256;
constexpr int64_t kSmemRows = 40000;       // keys of a row kept in shared memory up to this n
constexpr size_t kSmemBudget = 200u << 10;  // dynamic shared memory of the select kernel
constexpr size_t kTileBytes = 256u << 20;  // (R, n) FP32 tile budget

// distance key: the bits of d2 = max((sq_i + sq_j) - 2 dot, 0) (non-negative floats
// order like their bit patterns; -0 becomes 0)
__device__ __forceinline__ uint32_t dist_key(float dot, float sqi, float sqj) {
  const float d2 = fmaxf(__fsub_rn(__fadd_rn(sqi, sqj), __fmul_rn(2.f, dot)), 0.f);
  return __float_as_uint(d2) & 0x7fffffffu;
}

// exclusive prefix of flag over the block's threads, in thread order; *total = count
__device__ __forceinline__ int block_rank(bool flag, int* warp_cnt, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned b = __ballot_sync(0xffffffffu, flag);
  if (lane == 0) warp_cnt[warp] = __popc(b);
  __syncthreads();
  int before = 0, all = 0;
#pragma unroll
  for (int w = 0; w < kThreads / 32; ++w) {
    before += w < warp ? warp_cnt[w] : 0;
    all += warp_cnt[w];
  }
  __syncthreads();
  *total = all;
  return before + __popc(b & ((1u << lane) - 1u));
}

template <bool SMEM>
__global__ void __launch_bounds__(kThreads) select_kernel(const float* __restrict__ C, const float* __restrict__ sq,
                                                          const float* __restrict__ X, int64_t d, int64_t n,
                                                          int64_t q0, int k, int L, int P, int squared,
                                                          int32_t* __restrict__ out_idx,
                                                          float* __restrict__ out_dist) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  __shared__ unsigned hist[256];
  __shared__ int warp_cnt[kThreads / 32];
  __shared__ uint32_t s_pre, s_rank;
  __shared__ int s_cnt;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t row = blockIdx.x;
  const int64_t qi = q0 + row;
  const float* c = C + row * n;
  const float sqi = sq[qi];
  uint32_t* keys = reinterpret_cast<uint32_t*>(smem_raw);
  unsigned long long* buf =
      reinterpret_cast<unsigned long long*>(smem_raw + (SMEM ? ((size_t)n * 4 + 15) / 16 * 16 : 0));
  auto key_at = [&](int64_t j) -> uint32_t {
    if (SMEM) return keys[j];
    return j == qi ? 0xffffffffu : dist_key(c[j], sqi, sq[j]);
  };
  if (SMEM) {
    for (int64_t j = tid; j < n; j += kThreads) keys[j] = j == qi ? 0xffffffffu : dist_key(c[j], sqi, sq[j]);
    __syncthreads();
  }

  // radix select: the L-th smallest key (rank L), 8 bits a pass from the top
  uint32_t pre = 0u, msk = 0u, rank = (uint32_t)L;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int b = tid; b < 256; b += kThreads) hist[b] = 0u;
    __syncthreads();
    for (int64_t j = tid; j < n; j += kThreads) {
      const uint32_t x = key_at(j);
      if ((x & msk) == pre) atomicAdd(&hist[(x >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (warp == 0) {  // lane l owns bins 8l .. 8l + 7
      unsigned h[8], s = 0u;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        h[i] = hist[8 * lane + i];
        s += h[i];
      }
      unsigned incl = s;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      const unsigned excl = incl - s;
      if (excl < rank && rank <= incl) {
        unsigned cum = excl;
        int bin = 8 * lane + 7;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          if (cum + h[i] >= rank) {
            bin = 8 * lane + i;
            break;
          }
          cum += h[i];
        }
        s_pre = pre | ((uint32_t)bin << shift);
        s_rank = rank - cum;
      }
    }
    __syncthreads();
    pre = s_pre;
    rank = s_rank;
    msk |= 255u << shift;
    __syncthreads();
  }
  const uint32_t T = pre;           // the L-th smallest key
  const int take_eq = (int)rank;    // keys equal to T that belong to the L smallest

  // gather the keys below T (any order), then the first take_eq keys equal to T
  if (tid == 0) s_cnt = 0;
  __syncthreads();
  for (int64_t j = tid; j < n; j += kThreads) {
    const uint32_t x = key_at(j);
    if (x < T) buf[atomicAdd(&s_cnt, 1)] = ((unsigned long long)x << 32) | (uint32_t)j;
  }
  __syncthreads();
  const int nless = s_cnt;  // == L - take_eq
  int taken = 0;
  for (int64_t j0 = 0; j0 < n && taken < take_eq; j0 += kThreads) {
    const int64_t j = j0 + tid;
    const bool eq = j < n && key_at(j) == T;
    int total;
    const int r = block_rank(eq, warp_cnt, &total);
    if (eq && taken + r < take_eq) buf[nless + taken + r] = ((unsigned long long)T << 32) | (uint32_t)j;
    taken += total;
  }
  __syncthreads();
  // exact FP32 distances of the L candidates, one warp per candidate
  const float* xi = X + qi * d;
  for (int cand = warp; cand < L; cand += kThreads / 32) {
    const int64_t j = (int64_t)(uint32_t)buf[cand];
    const float* xj = X + j * d;
    float acc = 0.f;
    for (int64_t t = lane; t < d; t += 32) {
      const float diff = __fsub_rn(__ldg(xi + t), __ldg(xj + t));
      acc = fmaf(diff, diff, acc);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) buf[cand] = ((unsigned long long)__float_as_uint(acc) << 32) | (uint32_t)j;
  }
  for (int i = L + tid; i < P; i += kThreads) buf[i] = ~0ull;
  __syncthreads();

  // bitonic sort of P (key, index) words, ascending
  for (int size = 2; size <= P; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = tid; i < P / 2; i += kThreads) {
        const int lo = 2 * i - (i & (stride - 1));
        const int hi = lo + stride;
        const bool asc = (lo & size) == 0;
        const unsigned long long a = buf[lo], b = buf[hi];
        if ((a > b) == asc) {
          buf[lo] = b;
          buf[hi] = a;
        }
      }
      __syncthreads();
    }
  }
  for (int i = tid; i < k; i += kThreads) {
    const unsigned long long w = buf[i];
    const float d2 = __uint_as_float((uint32_t)(w >> 32));
    out_idx[row * k + i] = (int32_t)(uint32_t)w;
    out_dist[row * k + i] = squared ? d2 : sqrtf(d2);
  }
}

static int next_pow2(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}

static size_t keys_bytes(int64_t n) { return ((size_t)n * 4 + 15) / 16 * 16; }

// the row's keys are kept in shared memory when they fit next to the sort buffer
static bool keys_in_smem(int64_t n, int L) {
  return n <= kSmemRows && keys_bytes(n) + (size_t)next_pow2(L) * 8 <= kSmemBudget;
}

static size_t select_smem(int64_t n, int L) {
  const size_t pairs = (size_t)next_pow2(L) * 8;
  return keys_in_smem(n, L) ? keys_bytes(n) + pairs : pairs;
}

int plan(int64_t n, int64_t d, int k, int L, int64_t r0, int64_t m, void* ws, Plan& p) {
  if (k > kMaxK)
    return set_error(UMAPB_ERR_UNSUPPORTED, "knn_brute: k must be <= %d on the long-list path (got %d)", kMaxK, k);
  if (d > ((int64_t)1 << 20)) return set_error(UMAPB_ERR_UNSUPPORTED, "knn_brute: d above 2^20");
  if (n > 0x7fffffff) return set_error(UMAPB_ERR_UNSUPPORTED, "knn_brute: n above 2^31 - 1 on the long-list path");
  p.n = n;
  p.d = d;
  p.r0 = r0;
  p.m = m;
  p.k = k;
  p.L = L;
  p.kp = (int)((d + 63) / 64 * 64);
  int64_t R = (int64_t)(kTileBytes / ((size_t)n * 4)) / 128 * 128;
  if (R < 128) R = 128;
  p.R = R < m ? R : m;
  Carver c(ws);
  p.status = c.take<int32_t>(64);
  p.x3 = c.take<__nv_bfloat16>((size_t)n * 3 * p.kp);
  p.sq = c.take<float>((size_t)n);
  p.C = c.take<float>((size_t)p.R * n);
  p.bytes = c.bytes();
  return UMAPB_OK;
}

int run(const float* X, const Plan& p, int squared, int32_t* out_idx, float* out_dist, cudaStream_t stream) {
  const umapb_stream_t s = reinterpret_cast<umapb_stream_t>(stream);
  const size_t smem = select_smem(p.n, p.L);
  const int P = next_pow2(p.L);
  {
    static std::mutex mu;
    static size_t set_to[64][2] = {};
    int dev = 0;
    UMAPB_CUDA_TRY(cudaGetDevice(&dev), "knn_brute: device");
    std::lock_guard<std::mutex> lock(mu);
    const int v = keys_in_smem(p.n, p.L) ? 1 : 0;
    if (dev < 0 || dev >= 64 || set_to[dev][v] < smem) {
      UMAPB_CUDA_TRY(cudaFuncSetAttribute(v ? select_kernel<true> : select_kernel<false>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                     "knn_brute: select smem attribute");
      if (dev >= 0 && dev < 64) set_to[dev][v] = smem;
    }
  }
  UMAPB_CUDA_TRY(cudaMemsetAsync(p.status, 0, sizeof(int32_t), stream), "knn_brute: status reset");
  int rc;
  if ((rc = umapb_nnd_sqnorms(X, p.n, (int32_t)p.d, 0, p.sq, s))) return rc;
  if ((rc = umapb_split3(X, p.n, p.d, p.d, nullptr, 0, p.kp, p.x3, s))) return rc;
  const __nv_bfloat16* x3 = static_cast<const __nv_bfloat16*>(p.x3);
  for (int64_t b = 0; b < p.m; b += p.R) {
    const int64_t rows = p.m - b < p.R ? p.m - b : p.R;
    if ((rc = umapb_gemm_split3(x3 + (p.r0 + b) * 3 * (int64_t)p.kp, x3, (int32_t)rows, (int32_t)p.n, p.kp, 1, p.C,
                                (int32_t)p.n, p.status, s)))
      return rc;
    if (keys_in_smem(p.n, p.L))
      select_kernel<true><<<(unsigned)rows, kThreads, smem, stream>>>(p.C, p.sq, X, p.d, p.n, p.r0 + b, p.k, p.L, P,
                                                                      squared, out_idx + b * p.k, out_dist + b * p.k);
    else
      select_kernel<false><<<(unsigned)rows, kThreads, smem, stream>>>(p.C, p.sq, X, p.d, p.n, p.r0 + b, p.k, p.L, P,
                                                                       squared, out_idx + b * p.k, out_dist + b * p.k);
    UMAPB_LAUNCH_CHECK("knn_brute: select kernel");
    count_launches(1);
  }
  return UMAPB_OK;
}

}  // namespace knnx
}  // namespace umapb
