// Fuzzy simplicial set — replaces UMAP._fuzzy_simplicial_set, mlx_vis/_umap/umap.py:199-270.
//
// K1 weights:   one thread per row.  rho = max(min positive distance, 1e-8)
//               (umap.py:211-214); sigma by the reference's bisection
//               (umap.py:217-236: lo 1e-20, hi 1e3, sigma 1, 64 steps, target
//               log2 k over columns 1..k-1, converged when |sum - target| < 1e-5;
//               too high -> hi = sigma, sigma = (lo + sigma)/2; too low -> lo =
//               sigma, sigma = 2 sigma while hi >= 1e3 else (sigma + hi)/2), run in
//               double (or float, the reference's precision);
//               w = exp(-max(d - rho, 0) / max(sigma, 1e-10)) (umap.py:239).
// K2 symmetrise: one thread per directed edge (i, j): w' = weight of the first
//               entry of row j equal to i (what the reference's sorted-key
//               searchsorted finds, umap.py:241-260), w_sym = (w + w') - w w'
//               in float32 without contraction; grid max of w_sym.
// K3-K5 prune:  keep w_sym >= max / n_epochs (float32, umap.py:265-270) with an
//               order-preserving compaction (block counts, exclusive scan, write).
#include <math.h>

#include "common.cuh"
#include "scan.cuh"

namespace umapb {
namespace fuzzy {

constexpr int kBlock = 256;
constexpr int kEdgesPerBlock = 1024;  // 4 edges per thread in the prune kernels

template <class T>
__device__ __forceinline__ T dev_exp(T x);
template <>
__device__ __forceinline__ double dev_exp<double>(double x) { return exp(x); }
template <>
__device__ __forceinline__ float dev_exp<float>(float x) { return expf(x); }

template <class T>
__global__ void weights_kernel(const float* __restrict__ knn_dist, int64_t n, int k, float* __restrict__ w,
                               float* __restrict__ rho_out, float* __restrict__ sigma_out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* dr = knn_dist + i * k;
  T rho = (T)INFINITY;
  for (int j = 0; j < k; ++j) {
    const T v = (T)dr[j];
    if (v > (T)0 && v < rho) rho = v;
  }
  rho = rho > (T)1e-8 ? rho : (T)1e-8;  // max(rho, 1e-8); a row without positive distances keeps inf
  const T target = (T)log2((double)k);
  T lo = (T)1e-20, hi = (T)1e3, sigma = (T)1;
  for (int it = 0; it < 64; ++it) {
    T s = (T)0;
    for (int j = 1; j < k; ++j) {
      T ds = (T)dr[j] - rho;
      ds = ds > (T)0 ? ds : (T)0;
      s += dev_exp<T>(-ds / sigma);
    }
    const T diff = s - target;
    if ((diff < (T)0 ? -diff : diff) < (T)1e-5) break;
    if (s > target) {
      hi = sigma;
      sigma = (lo + sigma) / (T)2;
    } else if (s < target) {
      lo = sigma;
      sigma = hi >= (T)1e3 ? sigma * (T)2 : (sigma + hi) / (T)2;
    } else {
      break;  // NaN sums never converge; the reference keeps iterating without change
    }
  }
  const T sg = sigma > (T)1e-10 ? sigma : (T)1e-10;
  float* wr = w + i * k;
  for (int j = 0; j < k; ++j) {
    T ds = (T)dr[j] - rho;
    ds = ds > (T)0 ? ds : (T)0;
    wr[j] = (float)dev_exp<T>(-ds / sg);
  }
  if (rho_out) rho_out[i] = (float)rho;
  if (sigma_out) sigma_out[i] = (float)sigma;
}

__device__ __forceinline__ void atomic_max_nonneg(float* addr, float v) {
  // for non-negative floats the IEEE bit pattern orders like the value
  atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));
}

__global__ void symmetrize_kernel(const int32_t* __restrict__ knn_idx, const float* __restrict__ w, int64_t n,
                                  int k, float* __restrict__ w_sym, float* __restrict__ wmax) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float v = 0.f;
  if (e < n * k) {
    const int64_t i = e / k;
    const int32_t j = knn_idx[e];
    const float we = w[e];
    float wr = 0.f;
    if (j >= 0 && j < n) {
      const int32_t* rj = knn_idx + (int64_t)j * k;
      for (int p = 0; p < k; ++p) {
        if (rj[p] == (int32_t)i) {
          wr = w[(int64_t)j * k + p];
          break;
        }
      }
    }
    v = __fsub_rn(__fadd_rn(we, wr), __fmul_rn(we, wr));
    w_sym[e] = v;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(wmax, v);
}

__device__ __forceinline__ float prune_threshold(const float* wmax, int n_epochs) {
  return __fdiv_rn(*wmax, (float)n_epochs);
}

__global__ void prune_count_kernel(const float* __restrict__ w_sym, int64_t m, const float* __restrict__ wmax,
                                   int n_epochs, int32_t* __restrict__ block_counts) {
  __shared__ int warp_counts[kBlock / 32];
  const float thr = prune_threshold(wmax, n_epochs);
  const int64_t base = (int64_t)blockIdx.x * kEdgesPerBlock;
  int c = 0;
  for (int u = 0; u < kEdgesPerBlock / kBlock; ++u) {
    const int64_t e = base + u * kBlock + threadIdx.x;
    c += (e < m && w_sym[e] >= thr) ? 1 : 0;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) warp_counts[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int i = 0; i < kBlock / 32; ++i) t += warp_counts[i];
    block_counts[blockIdx.x] = t;
  }
}

__global__ void prune_write_kernel(const float* __restrict__ w_sym, const int32_t* __restrict__ knn_idx, int64_t m,
                                   int k, const float* __restrict__ wmax, int n_epochs,
                                   const int32_t* __restrict__ block_offsets, int32_t* __restrict__ rows,
                                   int32_t* __restrict__ cols, float* __restrict__ vals) {
  __shared__ int warp_base[kBlock / 32];
  __shared__ int running;
  const float thr = prune_threshold(wmax, n_epochs);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) running = block_offsets[blockIdx.x];
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kEdgesPerBlock;
  for (int u = 0; u < kEdgesPerBlock / kBlock; ++u) {
    const int64_t e = base + u * kBlock + threadIdx.x;
    const bool keep = e < m && w_sym[e] >= thr;
    const unsigned ballot = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) warp_base[warp] = __popc(ballot);
    __syncthreads();
    if (threadIdx.x == 0) {
      int s = running;
      for (int i = 0; i < kBlock / 32; ++i) {
        const int c = warp_base[i];
        warp_base[i] = s;
        s += c;
      }
      running = s;
    }
    __syncthreads();
    if (keep) {
      const int pos = warp_base[warp] + __popc(ballot & ((1u << lane) - 1u));
      rows[pos] = (int32_t)(e / k);
      cols[pos] = knn_idx[e];
      vals[pos] = w_sym[e];
    }
    __syncthreads();
  }
}

struct Layout {
  int32_t* status;
  float* w;
  float* w_sym;
  float* wmax;
  int32_t* block_counts;
  int64_t* scan_ws;  // scan_exclusive's block totals
  size_t bytes;
};

static Layout carve(void* ws, int64_t n, int k) {
  Carver c(ws);
  Layout l;
  l.status = c.take<int32_t>(64);
  l.w = c.take<float>((size_t)n * k);
  l.w_sym = c.take<float>((size_t)n * k);
  l.wmax = c.take<float>(64);
  l.block_counts = c.take<int32_t>((size_t)ceil_div(n * k, kEdgesPerBlock) + 1);
  l.scan_ws = c.take<int64_t>(kScanMaxBlocks);
  l.bytes = c.bytes();
  return l;
}

}  // namespace fuzzy
}  // namespace umapb

using namespace umapb;

extern "C" int umapb_fuzzy_workspace(int64_t n, int32_t k, size_t* bytes) {
  clear_error();
  UMAPB_REQUIRE(bytes, "bytes is null");
  UMAPB_REQUIRE(n >= 1 && k >= 1, "fuzzy: need n >= 1 and k >= 1");
  *bytes = fuzzy::carve(nullptr, n, k).bytes;
  return UMAPB_OK;
}

extern "C" int umapb_fuzzy(const int32_t* knn_idx, const float* knn_dist, int64_t n, int32_t k, int32_t n_epochs,
                           int32_t fp64_bisection, int32_t* rows, int32_t* cols, float* vals, int64_t* n_edges,
                           float* rho_out, float* sigma_out, void* workspace, size_t workspace_bytes,
                           umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(knn_idx && knn_dist && rows && cols && vals && n_edges, "fuzzy: null array argument");
  UMAPB_REQUIRE(n >= 1 && k >= 1, "fuzzy: need n >= 1 and k >= 1");
  UMAPB_REQUIRE(n_epochs >= 1, "fuzzy: n_epochs must be >= 1");
  UMAPB_REQUIRE(n * k < ((int64_t)1 << 31), "fuzzy: n*k must fit in int32");
  fuzzy::Layout l = fuzzy::carve(nullptr, n, k);
  if (!workspace || workspace_bytes < l.bytes)
    return set_error(UMAPB_ERR_WORKSPACE, "fuzzy: workspace of %zu bytes, need %zu", workspace_bytes, l.bytes);
  l = fuzzy::carve(workspace, n, k);
  const int64_t m = n * k;
  UMAPB_CUDA_TRY(cudaMemsetAsync(l.status, 0, 4, stream), "fuzzy: status reset");
  UMAPB_CUDA_TRY(cudaMemsetAsync(l.wmax, 0, 4, stream), "fuzzy: max reset");
  const unsigned row_blocks = (unsigned)ceil_div(n, fuzzy::kBlock);
  if (fp64_bisection)
    fuzzy::weights_kernel<double><<<row_blocks, fuzzy::kBlock, 0, stream>>>(knn_dist, n, k, l.w, rho_out, sigma_out);
  else
    fuzzy::weights_kernel<float><<<row_blocks, fuzzy::kBlock, 0, stream>>>(knn_dist, n, k, l.w, rho_out, sigma_out);
  UMAPB_LAUNCH_CHECK("fuzzy: weights kernel");
  fuzzy::symmetrize_kernel<<<(unsigned)ceil_div(m, fuzzy::kBlock), fuzzy::kBlock, 0, stream>>>(knn_idx, l.w, n, k,
                                                                                              l.w_sym, l.wmax);
  UMAPB_LAUNCH_CHECK("fuzzy: symmetrize kernel");
  const int64_t nb = ceil_div(m, fuzzy::kEdgesPerBlock);
  fuzzy::prune_count_kernel<<<(unsigned)nb, fuzzy::kBlock, 0, stream>>>(l.w_sym, m, l.wmax, n_epochs, l.block_counts);
  UMAPB_LAUNCH_CHECK("fuzzy: prune count kernel");
  scan_exclusive(l.block_counts, nb, n_edges, l.scan_ws, stream);
  UMAPB_LAUNCH_CHECK("fuzzy: scan kernel");
  fuzzy::prune_write_kernel<<<(unsigned)nb, fuzzy::kBlock, 0, stream>>>(l.w_sym, knn_idx, m, k, l.wmax, n_epochs,
                                                                       l.block_counts, rows, cols, vals);
  UMAPB_LAUNCH_CHECK("fuzzy: prune write kernel");
  count_launches(5);
  return UMAPB_OK;
}
