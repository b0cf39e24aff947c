// Dense FP32 products on the BF16 tensor cores and a stable key sort:
//
//   umapb_colmean       column means of a row-major FP32 matrix (FP64 partial sums,
//                       fixed summation order), the centring of PCA (umap.py:94-95)
//   umapb_split3        FP32 values x - mu (mu optional, per stored column) as three
//                       BF16 parts x0 + x1 + x2 side by side in rows of 3 kp, the
//                       operand layout of umapb_gemm_split3; `transpose` writes the
//                       stored columns as operand rows (X^T for the covariance)
//   umapb_sort_keys     stable ascending order of float keys (LSD radix sort, four
//                       8-bit passes): the row order NNDescent runs its rows in
//
// Split: x0 = bf16(x), x1 = bf16(x - x0), x2 = bf16(x - x0 - x1).  Both differences
// are exact in FP32 (each drops the leading 8 significant bits), so x0 + x1 + x2
// carries 24 significant bits of x; the products the split GEMM sums (x0 y0, x0 y1,
// x1 y0, x0 y2, x2 y0, x1 y1) miss only terms below 2^-24 |x y|.
#include <cuda_bf16.h>

#include "common.cuh"
#include "scan.cuh"

namespace umapb {
namespace linalg {

constexpr int kMeanRows = 1024;  // rows per FP64 partial sum of umapb_colmean

__global__ void colmean_partial_kernel(const float* __restrict__ S, int64_t rows, int64_t cols, int64_t lds,
                                       double* __restrict__ part) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  const int64_t r0 = (int64_t)blockIdx.y * kMeanRows;
  const int64_t r1 = r0 + kMeanRows < rows ? r0 + kMeanRows : rows;
  double s = 0.0;
  for (int64_t r = r0; r < r1; ++r) s += (double)S[r * lds + c];
  part[(int64_t)blockIdx.y * cols + c] = s;
}

__global__ void colmean_final_kernel(const double* __restrict__ part, int64_t chunks, int64_t rows, int64_t cols,
                                     float* __restrict__ mean) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  double s = 0.0;
  for (int64_t k = 0; k < chunks; ++k) s += part[k * cols + c];
  mean[c] = (float)(s / (double)rows);
}

__device__ __forceinline__ void split_value(float x, __nv_bfloat16& b0, __nv_bfloat16& b1, __nv_bfloat16& b2) {
  b0 = __float2bfloat16_rn(x);
  const float r1 = __fsub_rn(x, __bfloat162float(b0));
  b1 = __float2bfloat16_rn(r1);
  const float r2 = __fsub_rn(r1, __bfloat162float(b1));
  b2 = __float2bfloat16_rn(r2);
}

// operand row r = stored row r; columns c < cols hold S[r][c] - mu[c], [cols, kp) zeros.
// A thread splits 8 consecutive columns: two 16-byte loads (when S's rows and mu are
// 16-byte aligned and the group lies inside the row) and one 16-byte store per part.
__global__ void split_rows_kernel(const float* __restrict__ S, int64_t rows, int64_t cols, int64_t lds,
                                  const float* __restrict__ mu, int kp, int vec, __nv_bfloat16* __restrict__ out) {
  const int groups = kp / 8;
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t r = t / groups;
  const int c0 = (int)(t - r * groups) * 8;
  if (r >= rows) return;
  float x[8];
  const float* src = S + r * lds + c0;
  if (vec && c0 + 8 <= cols) {
    const float4 a = *reinterpret_cast<const float4*>(src), b = *reinterpret_cast<const float4*>(src + 4);
    x[0] = a.x, x[1] = a.y, x[2] = a.z, x[3] = a.w, x[4] = b.x, x[5] = b.y, x[6] = b.z, x[7] = b.w;
    if (mu) {
      const float4 ma = *reinterpret_cast<const float4*>(mu + c0), mb = *reinterpret_cast<const float4*>(mu + c0 + 4);
      const float m[8] = {ma.x, ma.y, ma.z, ma.w, mb.x, mb.y, mb.z, mb.w};
#pragma unroll
      for (int u = 0; u < 8; ++u) x[u] = __fsub_rn(x[u], m[u]);
    }
  } else {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int c = c0 + u;
      x[u] = c < cols ? (mu ? __fsub_rn(src[u], mu[c]) : src[u]) : 0.f;
    }
  }
  __align__(16) __nv_bfloat16 p0[8], p1[8], p2[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) split_value(x[u], p0[u], p1[u], p2[u]);
  uint4* o = reinterpret_cast<uint4*>(out + r * 3 * (int64_t)kp + c0);  // kp % 8 == 0: 16-byte aligned
  o[0] = *reinterpret_cast<const uint4*>(p0);
  o[kp / 8] = *reinterpret_cast<const uint4*>(p1);
  o[kp / 4] = *reinterpret_cast<const uint4*>(p2);
}

// operand row c = stored column c; columns r < rows hold S[r][c] - mu[c], [rows, kp)
// zeros.  32 x 32 tiles through shared memory: coalesced reads along c, writes along r.
__global__ void split_cols_kernel(const float* __restrict__ S, int64_t rows, int64_t cols, int64_t lds,
                                  const float* __restrict__ mu, int64_t kp, __nv_bfloat16* __restrict__ out) {
  __shared__ float tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.x * 32, c0 = (int64_t)blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int64_t r = r0 + j, c = c0 + threadIdx.x;
    float x = 0.f;
    if (r < rows && c < cols) x = mu ? __fsub_rn(S[r * lds + c], mu[c]) : S[r * lds + c];
    tile[j][threadIdx.x] = x;
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int64_t c = c0 + j, r = r0 + threadIdx.x;
    if (c >= cols || r >= kp) continue;
    __nv_bfloat16 b0, b1, b2;
    split_value(tile[threadIdx.x][j], b0, b1, b2);
    __nv_bfloat16* o = out + c * 3 * kp;
    o[r] = b0;
    o[kp + r] = b1;
    o[2 * kp + r] = b2;
  }
}

// ---- stable radix sort of float keys --------------------------------------------
constexpr int kSortTile = 1024;

// order-preserving unsigned image of a float; -0.0 maps with +0.0 (they compare
// equal, so the stable sort keeps them in index order)
__device__ __forceinline__ uint32_t f2ord(float f) {
  uint32_t u = __float_as_uint(f);
  if (u == 0x80000000u) u = 0u;
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void sort_init_kernel(const float* __restrict__ keys, int64_t n, int64_t stride, uint32_t* __restrict__ k0,
                                 int32_t* __restrict__ i0) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  k0[t] = f2ord(keys[t * stride]);
  i0[t] = (int32_t)t;
}

// counts[d * tiles + b] = keys of tile b whose digit is d
__global__ void __launch_bounds__(kSortTile) sort_hist_kernel(const uint32_t* __restrict__ k, int64_t n, int shift,
                                                              int32_t* __restrict__ counts) {
  __shared__ int32_t h[256];
  if (threadIdx.x < 256) h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t i = (int64_t)blockIdx.x * kSortTile + threadIdx.x;
  if (i < n) atomicAdd(&h[(k[i] >> shift) & 255u], 1);
  __syncthreads();
  if (threadIdx.x < 256) counts[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: a key's position is its digit's offset for this tile (scanned
// counts) + keys of the same digit in earlier warps + same digit in lower lanes.
__global__ void __launch_bounds__(kSortTile) sort_scatter_kernel(const uint32_t* __restrict__ kin,
                                                                 const int32_t* __restrict__ iin, int64_t n, int shift,
                                                                 const int32_t* __restrict__ offsets,
                                                                 uint32_t* __restrict__ kout,
                                                                 int32_t* __restrict__ iout) {
  __shared__ int32_t wc[kSortTile / 32][256];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int t = threadIdx.x; t < (kSortTile / 32) * 256; t += kSortTile) (&wc[0][0])[t] = 0;
  __syncthreads();
  const int64_t i = (int64_t)blockIdx.x * kSortTile + threadIdx.x;
  const bool valid = i < n;
  const uint32_t key = valid ? kin[i] : 0u;
  const int d = valid ? (int)((key >> shift) & 255u) : 256;
  const unsigned peers = __match_any_sync(0xffffffffu, d);
  const int rank = __popc(peers & ((1u << lane) - 1u));
  if (valid && rank == 0) wc[warp][d] = __popc(peers);
  __syncthreads();
  if (threadIdx.x < 256) {
    int32_t run = offsets[(int64_t)threadIdx.x * gridDim.x + blockIdx.x];
    for (int w = 0; w < kSortTile / 32; ++w) {
      const int32_t c = wc[w][threadIdx.x];
      wc[w][threadIdx.x] = run;
      run += c;
    }
  }
  __syncthreads();
  if (valid) {
    const int64_t pos = wc[warp][d] + rank;
    kout[pos] = key;
    iout[pos] = iin[i];
  }
}

struct SortLayout {
  uint32_t* k[2];
  int32_t* i[2];
  int32_t* counts;
  int64_t* total;
  int64_t* scan_ws;  // scan_exclusive's block totals
  size_t bytes;
};

static SortLayout sort_carve(void* ws, int64_t n) {
  Carver c(ws);
  SortLayout l;
  const int64_t tiles = ceil_div(n > 0 ? n : 1, kSortTile);
  for (int b = 0; b < 2; ++b) {
    l.k[b] = c.take<uint32_t>((size_t)(n > 0 ? n : 1));
    l.i[b] = c.take<int32_t>((size_t)(n > 0 ? n : 1));
  }
  l.counts = c.take<int32_t>((size_t)(256 * tiles));
  l.total = c.take<int64_t>(1);
  l.scan_ws = c.take<int64_t>(kScanMaxBlocks);
  l.bytes = c.bytes();
  return l;
}

}  // namespace linalg
}  // namespace umapb

using namespace umapb;

extern "C" int umapb_colmean_workspace(int64_t rows, int64_t cols, size_t* bytes) {
  clear_error();
  UMAPB_REQUIRE(bytes, "bytes is null");
  UMAPB_REQUIRE(rows >= 1 && cols >= 1, "colmean: need rows, cols >= 1");
  *bytes = (size_t)ceil_div(rows, linalg::kMeanRows) * (size_t)cols * sizeof(double) + 256;
  return UMAPB_OK;
}

extern "C" int umapb_colmean(const float* S, int64_t rows, int64_t cols, int64_t lds, float* mean, void* workspace,
                             size_t workspace_bytes, umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(S && mean, "colmean: null argument");
  UMAPB_REQUIRE(rows >= 1 && cols >= 1 && lds >= cols, "colmean: need rows, cols >= 1 and lds >= cols");
  const int64_t chunks = ceil_div(rows, linalg::kMeanRows);
  const size_t need = (size_t)chunks * (size_t)cols * sizeof(double);
  if (!workspace || workspace_bytes < need)
    return set_error(UMAPB_ERR_WORKSPACE, "colmean: workspace of %zu bytes, need %zu", workspace_bytes, need);
  UMAPB_REQUIRE(chunks < 65536, "colmean: too many rows");
  double* part = static_cast<double*>(workspace);
  linalg::colmean_partial_kernel<<<dim3((unsigned)ceil_div(cols, 256), (unsigned)chunks), 256, 0, stream>>>(
      S, rows, cols, lds, part);
  linalg::colmean_final_kernel<<<(unsigned)ceil_div(cols, 256), 256, 0, stream>>>(part, chunks, rows, cols, mean);
  UMAPB_LAUNCH_CHECK("colmean kernels");
  count_launches(2);
  return UMAPB_OK;
}

extern "C" int umapb_split3(const float* S, int64_t rows, int64_t cols, int64_t lds, const float* mu,
                            int32_t transpose, int32_t kp, void* out, umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(S && out, "split3: null argument");
  UMAPB_REQUIRE(rows >= 1 && cols >= 1 && lds >= cols, "split3: need rows, cols >= 1 and lds >= cols");
  UMAPB_REQUIRE(kp >= 64 && kp % 64 == 0, "split3: kp must be a positive multiple of 64");
  UMAPB_REQUIRE(kp >= (transpose ? rows : cols), "split3: kp must cover the operand's K extent");
  __nv_bfloat16* o = static_cast<__nv_bfloat16*>(out);
  if (!transpose) {
    const int64_t total = rows * (kp / 8);
    const int vec = (reinterpret_cast<uintptr_t>(S) & 15) == 0 && lds % 4 == 0 &&
                    (!mu || (reinterpret_cast<uintptr_t>(mu) & 15) == 0);
    linalg::split_rows_kernel<<<(unsigned)ceil_div(total, 256), 256, 0, stream>>>(S, rows, cols, lds, mu, kp, vec,
                                                                                   o);
  } else {
    UMAPB_REQUIRE(ceil_div(cols, 32) < 65536, "split3: too many columns to transpose");
    linalg::split_cols_kernel<<<dim3((unsigned)ceil_div(kp, 32), (unsigned)ceil_div(cols, 32)), dim3(32, 8), 0,
                                stream>>>(S, rows, cols, lds, mu, kp, o);
  }
  UMAPB_LAUNCH_CHECK("split3 kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_sort_keys_workspace(int64_t n, size_t* bytes) {
  clear_error();
  UMAPB_REQUIRE(bytes, "bytes is null");
  UMAPB_REQUIRE(n >= 0 && n < ((int64_t)1 << 31), "sort_keys: need 0 <= n < 2^31");
  *bytes = linalg::sort_carve(nullptr, n).bytes;
  return UMAPB_OK;
}

extern "C" int umapb_sort_keys(const float* keys, int64_t n, int64_t stride, int32_t* order, void* workspace,
                               size_t workspace_bytes,
                               umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(n >= 0 && n < ((int64_t)1 << 31), "sort_keys: need 0 <= n < 2^31");
  if (n == 0) return UMAPB_OK;
  UMAPB_REQUIRE(keys && order, "sort_keys: null argument");
  UMAPB_REQUIRE(stride >= 1, "sort_keys: stride must be >= 1");
  linalg::SortLayout l = linalg::sort_carve(nullptr, n);
  if (!workspace || workspace_bytes < l.bytes)
    return set_error(UMAPB_ERR_WORKSPACE, "sort_keys: workspace of %zu bytes, need %zu", workspace_bytes, l.bytes);
  l = linalg::sort_carve(workspace, n);
  const int64_t tiles = ceil_div(n, linalg::kSortTile);
  linalg::sort_init_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, stream>>>(keys, n, stride, l.k[0], l.i[0]);
  for (int pass = 0; pass < 4; ++pass) {
    const int src = pass & 1, dst = src ^ 1;
    linalg::sort_hist_kernel<<<(unsigned)tiles, linalg::kSortTile, 0, stream>>>(l.k[src], n, 8 * pass, l.counts);
    scan_exclusive(l.counts, 256 * tiles, l.total, l.scan_ws, stream);
    int32_t* iout = pass == 3 ? order : l.i[dst];
    linalg::sort_scatter_kernel<<<(unsigned)tiles, linalg::kSortTile, 0, stream>>>(
        l.k[src], l.i[src], n, 8 * pass, l.counts, l.k[dst], iout);
  }
  UMAPB_LAUNCH_CHECK("sort_keys kernels");
  count_launches(1 + 4 * 3);
  return UMAPB_OK;
}

namespace umapb {
namespace linalg {
__global__ void sum_slices_kernel(const float* __restrict__ C, int slices, int64_t count, float scale,
                                  float* __restrict__ out) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  double s = 0.0;  // FP64: the slices' FP32 partial sums add without further rounding drift
  for (int z = 0; z < slices; ++z) s += (double)C[(int64_t)z * count + t];
  out[t] = (float)(s * (double)scale);
}
}  // namespace linalg
}  // namespace umapb

extern "C" int umapb_sum_slices(const float* C, int32_t slices, int64_t count, float scale, float* out,
                                umapb_stream_t stream_) {
  clear_error();
  UMAPB_REQUIRE(C && out, "sum_slices: null argument");
  UMAPB_REQUIRE(slices >= 1 && count >= 0, "sum_slices: need slices >= 1 and count >= 0");
  if (count == 0) return UMAPB_OK;
  linalg::sum_slices_kernel<<<(unsigned)ceil_div(count, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream_)>>>(
      C, slices, count, scale, out);
  UMAPB_LAUNCH_CHECK("sum_slices kernel");
  count_launches(1);
  return UMAPB_OK;
}
