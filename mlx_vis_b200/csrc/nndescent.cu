// NNDescent kNN graph — replaces mlx_vis/_nndescent/nndescent.py:34-486 and 573-641.
//
// The host (Python) keeps the reference's control flow (random init and
// projections from NumPy's global stream, per-iteration mc/j_nn from the update
// fraction, full vs converging path, FP16 iterations 1-4, low-dimensional
// iterations 0-1, FP32 recompute after iteration 4).  These kernels do the data
// work of one iteration:
//
// reverse candidates (nndescent.py:406-436): slot p of row j = p-th smallest
//   source i with j in knn(i); empty slots hold 0 (the reference's zero padding).
//   Bucket fill with atomics, then one warp sorts each bucket: deterministic.
// row update (nndescent.py:241-280 full path, 103-220 converging path), one warp
//   per row:
//   1. candidate row = [current k | nn-of-nn (mc_new sources x first j_nn of
//      their rows) | reverse k]; on the converging path the sources are the
//      row's NEW neighbours first (stable), and rows with no NEW flag are copied.
//   2. duplicates: the first occurrence in that order survives (a shared-memory
//      hash set per warp; equal ids inside one 32-wide chunk resolved with
//      __match_any_sync) — what the reference's stable sort by id keeps.
//   3. distances max(sq_i + sq_c - 2 x_i.x_c, 0) only for surviving candidates
//      that need one: stored distances are reused for current neighbours unless
//      the iteration recomputes them; FP16 iterations round the FP32-accumulated
//      dot product to FP16 like _gather_dists_half.  Self and duplicates get 1e30.
//   4. the k smallest (distance, id) pairs, kept as a warp-distributed sorted list
//      (ballot finds the slot, shfl_up shifts), written with the positional
//      change flags and a global count of changes (nndescent.py:381-385).
#include <cuda_fp16.h>
#include <math.h>

#include <mutex>

#include "common.cuh"
#include "nnd_wide.cuh"
#include "scan.cuh"

namespace umapb {
namespace nnd {

constexpr float kBig = 1e30f;
constexpr int kWarps = 4;  // warps per block in the row kernels

__device__ __forceinline__ bool key_lt(float a, int ia, float b, int ib) {
  return a < b || (a == b && ia < ib);
}

// ---- distance helpers --------------------------------------------------------
template <class T>
__device__ __forceinline__ float to_f(T v);
template <>
__device__ __forceinline__ float to_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ float to_f<__half>(__half v) { return __half2float(v); }

// dot products of x (shared memory copy of row i) with up to 4 rows of X, summed
// over the warp; every lane gets the totals
template <class T>
__device__ __forceinline__ void dot4(const T* __restrict__ X, const T* xs, int dd, const int (&c)[4], int cnt,
                                     int lane, float (&out)[4]) {
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  constexpr int V = 16 / sizeof(T);  // elements per 16-byte vector
  const bool vec = (dd % V) == 0 && (reinterpret_cast<uintptr_t>(X) & 15) == 0;
  if (vec) {
    const int nv = dd / V;
    for (int t = lane; t < nv; t += 32) {
      const uint4 a4 = reinterpret_cast<const uint4*>(xs)[t];
      const T* a = reinterpret_cast<const T*>(&a4);
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (u < cnt) {
          const uint4 b4 = __ldg(reinterpret_cast<const uint4*>(X + (int64_t)c[u] * dd) + t);
          const T* bb = reinterpret_cast<const T*>(&b4);
#pragma unroll
          for (int e = 0; e < V; ++e) acc[u] = fmaf(to_f<T>(a[e]), to_f<T>(bb[e]), acc[u]);
        }
      }
    }
  } else {
    for (int t = lane; t < dd; t += 32) {
      const float a = to_f<T>(xs[t]);
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (u < cnt) acc[u] = fmaf(a, to_f<T>(X[(int64_t)c[u] * dd + t]), acc[u]);
    }
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[u] += __shfl_xor_sync(0xffffffffu, acc[u], o);
    out[u] = acc[u];
  }
}

__device__ __forceinline__ float d2_from_dot(float sq_i, float sq_c, float dot, bool half_round) {
  if (half_round) dot = __half2float(__float2half_rn(dot));
  return fmaxf(__fsub_rn(__fadd_rn(sq_i, sq_c), __fmul_rn(2.0f, dot)), 0.0f);
}

// ascending bitonic sort of one (distance, id) key per lane across the warp
__device__ __forceinline__ void warp_sort_keys(float& d, int& id, int lane) {
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const float od = __shfl_xor_sync(0xffffffffu, d, stride);
      const int oi = __shfl_xor_sync(0xffffffffu, id, stride);
      const bool lower = (lane & stride) == 0, asc = (lane & size) == 0;
      const bool take = (lower == asc) ? key_lt(od, oi, d, id) : key_lt(d, id, od, oi);
      if (take) {
        d = od;
        id = oi;
      }
    }
  }
}

// ascending order of a bitonic sequence held one key per lane
__device__ __forceinline__ void warp_bitonic_clean(float& d, int& id, int lane) {
#pragma unroll
  for (int stride = 16; stride > 0; stride >>= 1) {
    const float od = __shfl_xor_sync(0xffffffffu, d, stride);
    const int oi = __shfl_xor_sync(0xffffffffu, id, stride);
    const bool take = (lane & stride) == 0 ? key_lt(od, oi, d, id) : key_lt(d, id, od, oi);
    if (take) {
      d = od;
      id = oi;
    }
  }
}

// Inserts (d, id) into the warp-distributed ascending list (lane l holds entry l).
// Inserts (d, id) into the warp-distributed ascending list (lane l holds entry l).
__device__ __forceinline__ void list_insert(float& lv, int& li, float d, int id, int k, int lane) {
  const int pos = __popc(__ballot_sync(0xffffffffu, lane < k && key_lt(lv, li, d, id)));
  const float up_v = __shfl_up_sync(0xffffffffu, lv, 1);
  const int up_i = __shfl_up_sync(0xffffffffu, li, 1);
  if (lane < k) {
    if (lane > pos) {
      lv = up_v;
      li = up_i;
    } else if (lane == pos) {
      lv = d;
      li = id;
    }
  }
}

// ---- small kernels -------------------------------------------------------------
template <class T>
__global__ void sqnorm_kernel(const T* __restrict__ X, int64_t n, int dd, float* __restrict__ sq) {
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  float acc = 0.f;
  for (int t = lane; t < dd; t += 32) {
    const float v = to_f<T>(X[row * dd + t]);
    acc = fmaf(v, v, acc);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) sq[row] = acc;
}

// FP16 copy of (n, dd) FP32 rows into rows of pitch ldh >= dd, zero padded
__global__ void to_half_kernel(const float* __restrict__ X, int64_t n, int dd, int ldh, __half* __restrict__ H) {
  const int64_t m = n * ldh;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / ldh;
    const int c = (int)(t - r * ldh);
    H[t] = c < dd ? __float2half_rn(X[r * dd + c]) : __float2half_rn(0.0f);
  }
}

// d2 of each row to its k listed neighbours (FP32, full space), optionally sorted
// ascending by (distance, id) — _gather_dists (nndescent.py:573-612) and the sort
// after the random init (nndescent.py:63-65).
__global__ void gather_rows_kernel(const float* __restrict__ X, const float* __restrict__ sq, int64_t n, int dd,
                                   int32_t* __restrict__ idx, float* __restrict__ dist, int k, int sort_rows) {
  extern __shared__ float xs_all[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * kWarps + warp;
  if (row >= n) return;
  float* xs = xs_all + warp * dd;
  for (int t = lane; t < dd; t += 32) xs[t] = X[row * dd + t];
  __syncwarp();
  const float sqi = sq[row];
  float my_d = kBig;
  int my_i = 0x7fffffff;
  for (int p0 = 0; p0 < k; p0 += 4) {
    int c[4];
    const int cnt = min(4, k - p0);
    for (int u = 0; u < 4; ++u) c[u] = u < cnt ? idx[row * k + p0 + u] : 0;
    float dots[4];
    dot4<float>(X, xs, dd, c, cnt, lane, dots);
    for (int u = 0; u < cnt; ++u) {
      const float d2 = d2_from_dot(sqi, sq[c[u]], dots[u], false);
      if (lane == p0 + u) {
        my_d = d2;
        my_i = c[u];
      }
    }
  }
  if (sort_rows) warp_sort_keys(my_d, my_i, lane);  // k <= 32 (distance, id) pairs, one per lane
  if (lane < k) {
    idx[row * k + lane] = my_i;
    dist[row * k + lane] = my_d;
  }
}

// The pairs (i, j = idx[i][p]) of rows i < r1 whose later row max(i, j) lies in
// [r0, r1): launched once per row block of an upload in row order, every pair is
// computed once, as soon as both of its rows are on the device, with the same
// expression and summation order as gather_rows_kernel.  idx is not changed and the
// other entries of dist are left as they are; sort_rows_kernel sorts after the last
// block.  k <= 32.
__global__ void gather_pairs_kernel(const float* __restrict__ X, const float* __restrict__ sq, int dd,
                                    const int32_t* __restrict__ idx, float* __restrict__ dist, int k, int64_t r0,
                                    int64_t r1) {
  extern __shared__ float xs_all[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * kWarps + warp;
  if (row >= r1) return;
  const int my_j = lane < k ? idx[row * k + lane] : 0;
  const int64_t later = my_j > row ? (int64_t)my_j : row;
  unsigned todo = __ballot_sync(0xffffffffu, lane < k && later >= r0 && later < r1);
  if (!todo) return;
  float* xs = xs_all + warp * dd;
  for (int t = lane; t < dd; t += 32) xs[t] = X[row * dd + t];
  __syncwarp();
  const float sqi = sq[row];
  while (todo) {  // up to four positions per step, in ascending order (warp-uniform)
    int pos[4], c[4];
    int cnt = 0;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      pos[u] = todo ? __ffs(todo) - 1 : 0;
      if (todo) {
        todo &= todo - 1;
        ++cnt;
      }
      c[u] = __shfl_sync(0xffffffffu, my_j, pos[u]);
    }
    float dots[4];
    dot4<float>(X, xs, dd, c, cnt, lane, dots);
    for (int u = 0; u < cnt; ++u)
      if (lane == pos[u]) dist[row * k + lane] = d2_from_dot(sqi, sq[c[u]], dots[u], false);
  }
}

// Each row of (dist, idx) sorted by (distance, id), k <= 32 entries, one warp per row.
__global__ void sort_rows_kernel(int32_t* __restrict__ idx, float* __restrict__ dist, int64_t n, int k) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * kWarps + warp;
  if (row >= n) return;
  float d = lane < k ? dist[row * k + lane] : kBig;
  int i = lane < k ? idx[row * k + lane] : 0x7fffffff;
  warp_sort_keys(d, i, lane);
  if (lane < k) {
    idx[row * k + lane] = i;
    dist[row * k + lane] = d;
  }
}

// ---- reverse candidates ----------------------------------------------------------
__global__ void indegree_kernel(const int32_t* __restrict__ idx, int64_t m, int32_t* __restrict__ deg) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&deg[idx[t]], 1);
}

__global__ void bucket_fill_kernel(const int32_t* __restrict__ idx, int64_t m, int k, const int32_t* __restrict__ off,
                                   int32_t* __restrict__ fill, int32_t* __restrict__ bucket) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    const int j = idx[t];
    const int p = atomicAdd(&fill[j], 1);
    bucket[off[j] + p] = (int32_t)(t / k);
  }
}

// rev[j][p] = p-th smallest source in j's bucket, 0 when the bucket is shorter.
// Bucket entries hold the source row shifted left by `shift` bits (0 for the
// reverse buckets, 5 for the join's (row, position) entries); deg == nullptr
// takes the bucket sizes from the offsets (off[n] = total).
//
// A bucket of more than 32 entries (or k > 32), one warp: the sorted multiset of j's
// sources, first k of it.  Each pass emits the previous source again while it has
// unused copies (a row that lists j twice), else the next larger source; once the
// bucket is exhausted the remaining slots stay 0, as the reference's scatter into
// zeros leaves them.
__device__ void bucket_select_long(const int32_t* __restrict__ b, int cnt, int k, int shift,
                                   int32_t* __restrict__ out, int lane) {
  int prev = -1, used = 0, copies = 0;
  for (int p = 0; p < k; ++p) {
    int o;
    if (prev >= 0 && used < copies) {
      o = prev;
      ++used;
    } else {
      int best = 0x7fffffff;
      for (int t = lane; t < cnt; t += 32) {
        const int s = b[t] >> shift;
        if (s > prev && s < best) best = s;
      }
#pragma unroll
      for (int q = 16; q > 0; q >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, q));
      if (best == 0x7fffffff) {
        for (int q = p + lane; q < k; q += 32) out[q] = 0;
        return;
      }
      int c = 0;
      for (int t = lane; t < cnt; t += 32) c += (b[t] >> shift) == best ? 1 : 0;
#pragma unroll
      for (int q = 16; q > 0; q >>= 1) c += __shfl_xor_sync(0xffffffffu, c, q);
      o = best;
      prev = best;
      copies = c;
      used = 1;
    }
    if (lane == 0) out[p] = o;
  }
}

// kSelRows consecutive rows per warp: their offsets come in one load per lane and
// their bucket entries (up to 32 each) in kSelRows loads issued together, so a warp
// waits for two round trips per kSelRows rows instead of per row.  A bucket of at
// most 32 entries (the common case: the mean in-degree is k) is sorted across the
// warp by a bitonic network; lane p then holds the p-th smallest source.
constexpr int kSelRows = 4;
__global__ void bucket_select_kernel(const int32_t* __restrict__ bucket, const int32_t* __restrict__ off,
                                     const int32_t* __restrict__ deg, int64_t n, int k, int shift,
                                     int32_t* __restrict__ rev) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t j0 = ((int64_t)blockIdx.x * kWarps + warp) * kSelRows;
  if (j0 >= n) return;
  // lane r < kSelRows: off[j0 + r] (and deg); without deg lane kSelRows also loads the
  // next row's offset (off[n] is the total there)
  const int64_t jl = j0 + lane;
  const int span = deg ? kSelRows : kSelRows + 1;
  const int64_t lim = deg ? n : n + 1;
  const int o = (lane < span && jl < lim) ? off[jl] : 0;
  const int dg = (deg && lane < kSelRows && jl < n) ? deg[jl] : 0;
  int start[kSelRows], cnt[kSelRows], v[kSelRows];
#pragma unroll
  for (int r = 0; r < kSelRows; ++r) {
    start[r] = __shfl_sync(0xffffffffu, o, r);
    const int nxt = __shfl_sync(0xffffffffu, o, r + 1);
    const int c = deg ? __shfl_sync(0xffffffffu, dg, r) : nxt - start[r];
    cnt[r] = j0 + r < n ? c : -1;  // -1: past the last row
  }
#pragma unroll
  for (int r = 0; r < kSelRows; ++r)
    v[r] = (cnt[r] >= 0 && cnt[r] <= 32 && lane < cnt[r]) ? (bucket[start[r] + lane] >> shift) : 0x7fffffff;
#pragma unroll
  for (int r = 0; r < kSelRows; ++r) {
    if (cnt[r] < 0) break;  // warp-uniform: every lane holds the same counts
    const int64_t j = j0 + r;
    if (cnt[r] <= 32 && k <= 32) {
      int x = v[r];
      for (int size = 2; size <= 32; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
          const int y = __shfl_xor_sync(0xffffffffu, x, stride);
          const bool lower = (lane & stride) == 0, asc = (lane & size) == 0;
          x = (lower == asc) ? min(x, y) : max(x, y);
        }
      }
      if (lane < k) rev[j * k + lane] = lane < cnt[r] ? x : 0;
    } else {
      bucket_select_long(bucket + start[r], cnt[r], k, shift, rev + j * k, lane);
    }
  }
}

// ---- distance phase helpers ------------------------------------------------------
// FP16 rows (pitch a multiple of 8 halves, zero padded): 16 candidates per warp
// step on the tensor cores.  mma.m16n8k16 multiplies A (16 candidate rows x 16
// dims) by B (16 dims x 8 columns, every column the query row), FP32 accumulate.
// Thread (g = lane / 4, c = lane % 4) supplies A for rows g and g + 8 and B for
// column g at the logical k positions {2c, 2c+1, 2c+8, 2c+9}; it loads 16-byte
// chunks c + 4s of the rows and of the query, and maps their halves 0-3 to one
// mma and 4-7 to the next.  The k positions of A and B come from the same physical
// dims (the map depends on c alone), so every column of D is the dot product.
__device__ __forceinline__ void mma_f16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                        uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// d2 for the candidates todo[0, n_todo) of one row, FP16 space: cd[t] for each.
// Two independent 16-candidate tiles per step keep four row loads in flight per
// thread.
__device__ __forceinline__ void dists_f16(const __half* __restrict__ X, int ldx, const __half* xs, const float* sqd,
                                          float sqi, int64_t row, const int32_t* cid, const uint16_t* todo,
                                          int n_todo, float* cd, int lane) {
  const int V = ldx / 8;  // 16-byte chunks per row
  const int S = (V + 3) / 4;
  const int g = lane >> 2, c = lane & 3;
  const uint4* xq = reinterpret_cast<const uint4*>(xs);
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
  for (int p0 = 0; p0 < n_todo; p0 += 32) {
    int t[4], cc[4];
    bool v[4];
    const uint4* r[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {  // tile rows g, g + 8 (tile 0) and g + 16, g + 24 (tile 1)
      const int p = p0 + g + 8 * u;
      v[u] = p < n_todo;
      t[u] = v[u] ? todo[p] : 0;
      cc[u] = v[u] ? cid[t[u]] : (int)row;
      r[u] = reinterpret_cast<const uint4*>(X + (int64_t)cc[u] * ldx);
    }
    float d0[4] = {0.f, 0.f, 0.f, 0.f}, d1[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 2
    for (int st = 0; st < S; ++st) {
      const int q = c + 4 * st;
      const bool in = q < V;
      uint4 A[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) A[u] = (in && v[u]) ? __ldg(r[u] + q) : zero;
      const uint4 B = in ? xq[q] : zero;
      mma_f16(d0, A[0].x, A[1].x, A[0].y, A[1].y, B.x, B.y);
      mma_f16(d0, A[0].z, A[1].z, A[0].w, A[1].w, B.z, B.w);
      mma_f16(d1, A[2].x, A[3].x, A[2].y, A[3].y, B.x, B.y);
      mma_f16(d1, A[2].z, A[3].z, A[2].w, A[3].w, B.z, B.w);
    }
    // d0[0]: row g, d0[2]: row g + 8, d1[0]: row g + 16, d1[2]: row g + 24 (every column
    // holds the same dot); lane c stores row g + 8c
    const float dot = c == 0 ? d0[0] : c == 1 ? d0[2] : c == 2 ? d1[0] : d1[2];
    const int tt = c == 0 ? t[0] : c == 1 ? t[1] : c == 2 ? t[2] : t[3];
    const int cs = c == 0 ? cc[0] : c == 1 ? cc[1] : c == 2 ? cc[2] : cc[3];
    const bool vs = c == 0 ? v[0] : c == 1 ? v[1] : c == 2 ? v[2] : v[3];
    if (vs) cd[tt] = d2_from_dot(sqi, sqd[cs], dot, true);
  }
}

// FP32 rows: G lanes per candidate, each lane group working on two candidates at
// once (2 * 32 / G per warp step), float4 loads when the pitch allows, a
// log2(G)-step shuffle reduction.
template <bool VEC>
__device__ __forceinline__ void dists_f32(const float* __restrict__ X, int dd, int ldx, const float* xs,
                                          const float* sqd, float sqi, int64_t row, const int32_t* cid,
                                          const uint16_t* todo, int n_todo, float* cd, int lane, int G) {
  const int C = 32 / G;
  const int j = lane & (G - 1), slot = lane / G;
  for (int p0 = 0; p0 < n_todo; p0 += 2 * C) {
    const int pa = p0 + slot, pb = p0 + C + slot;
    const bool va = pa < n_todo, vb = pb < n_todo;
    const int ta = va ? todo[pa] : 0, tb = vb ? todo[pb] : 0;
    const int ca = va ? cid[ta] : (int)row, cb = vb ? cid[tb] : (int)row;
    float acc_a = 0.f, acc_b = 0.f;
    if (VEC) {
      const float4* ra = reinterpret_cast<const float4*>(X + (int64_t)ca * ldx);
      const float4* rb = reinterpret_cast<const float4*>(X + (int64_t)cb * ldx);
      const float4* xp = reinterpret_cast<const float4*>(xs);
      const int V = dd / 4;
#pragma unroll 4
      for (int q = j; q < V; q += G) {
        const float4 x = xp[q];
        const float4 a4 = __ldg(ra + q);
        const float4 b4 = vb ? __ldg(rb + q) : make_float4(0.f, 0.f, 0.f, 0.f);
        acc_a = fmaf(x.x, a4.x, acc_a);
        acc_a = fmaf(x.y, a4.y, acc_a);
        acc_a = fmaf(x.z, a4.z, acc_a);
        acc_a = fmaf(x.w, a4.w, acc_a);
        acc_b = fmaf(x.x, b4.x, acc_b);
        acc_b = fmaf(x.y, b4.y, acc_b);
        acc_b = fmaf(x.z, b4.z, acc_b);
        acc_b = fmaf(x.w, b4.w, acc_b);
      }
    } else {
      const float* ra = X + (int64_t)ca * ldx;
      const float* rb = X + (int64_t)cb * ldx;
      for (int q = j; q < dd; q += G) {
        const float x = xs[q];
        acc_a = fmaf(x, __ldg(ra + q), acc_a);
        if (vb) acc_b = fmaf(x, __ldg(rb + q), acc_b);
      }
    }
    for (int o = G >> 1; o > 0; o >>= 1) {
      acc_a += __shfl_xor_sync(0xffffffffu, acc_a, o);
      acc_b += __shfl_xor_sync(0xffffffffu, acc_b, o);
    }
    if (va && j == 0) cd[ta] = d2_from_dot(sqi, sqd[ca], acc_a, false);
    if (vb && j == 1 % G) cd[tb] = d2_from_dot(sqi, sqd[cb], acc_b, false);
  }
}


// ---- blocked join of the nn-of-nn candidates (full-path iterations) ---------------
// Row i's nn-of-nn candidates are the first j_nn neighbours of each of its first mc
// neighbours (its sources).  Grouped by source s, they form one dense block: every
// row i that lists s at a position p < mc, against the columns [s, first j_nn
// neighbours of s].  One warp per source computes that block; block (i, p) x
// column 0 is the current-neighbour distance d(i, s) -> curd[i][p], column 1 + j
// the candidate at the reference's column k + p*j_nn + j -> nnbuf[i][p*j_nn + j].
// One warp takes one 16-entry chunk of a bucket against all its columns.
// Each output slot belongs to exactly one (source, entry, column), so the buffers
// are written without atomics and the result does not depend on the bucket order.
// A row's vector is read once per source that lists it instead of once per
// candidate: about mc + 1 + j_nn row reads per row instead of ~k + mc*j_nn + k.

// entries: (i, p) with p < mc, bucketed by s = idx[i][p]; encoded i * 32 + p
// The source of entry (i, p): idx[i][p], or srcs[i][p] when a source list is given
// (negative: no source)
__device__ __forceinline__ int entry_source(const int32_t* __restrict__ idx, const int32_t* __restrict__ srcs,
                                            int64_t t, int k, int mc) {
  return srcs ? srcs[t] : idx[(t / mc) * k + (t % mc)];
}

__global__ void src_count_kernel(const int32_t* __restrict__ idx, const int32_t* __restrict__ srcs, int64_t n, int k,
                                 int mc, int32_t* __restrict__ cnt) {
  const int64_t m = n * mc;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    const int sidx = entry_source(idx, srcs, t, k, mc);
    if (sidx >= 0) atomicAdd(&cnt[sidx], 1);
  }
}

__global__ void src_fill_kernel(const int32_t* __restrict__ idx, const int32_t* __restrict__ srcs, int64_t n, int k,
                                int mc, const int32_t* __restrict__ off, int32_t* __restrict__ fill,
                                int32_t* __restrict__ entries) {
  const int64_t m = n * mc;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    const int sidx = entry_source(idx, srcs, t, k, mc);
    if (sidx < 0) continue;
    const int64_t i = t / mc;
    const int p = (int)(t % mc);
    entries[off[sidx] + atomicAdd(&fill[sidx], 1)] = (int32_t)(i * 32 + p);
  }
}

// The converging path's sources (nndescent.py:103-107): the first mc of each row's
// neighbours in NEW-first stable order, or none (-1) for a row without a NEW one
// (its list stays as it is).  One warp per row, the row kernel's ordering rule.
__global__ void new_sources_kernel(const int32_t* __restrict__ idx, const uint8_t* __restrict__ flags, int64_t n,
                                   int k, int mc, int32_t* __restrict__ srcs) {
  const int lane = threadIdx.x & 31;
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (row >= n) return;
  const bool f = lane < k && flags[row * k + lane];
  const unsigned fb = __ballot_sync(0xffffffffu, f);
  if (fb == 0) {
    for (int p = lane; p < mc; p += 32) srcs[row * mc + p] = -1;
    return;
  }
  const unsigned lt = (1u << lane) - 1u;
  const unsigned ob = __ballot_sync(0xffffffffu, lane < k && !f);
  const int pos = f ? __popc(fb & lt) : __popc(fb) + __popc(ob & lt);
  if (lane < k && pos < mc) srcs[row * mc + pos] = idx[row * k + lane];
}

// work items: 16-entry chunks of each bucket (hub sources, listed by hundreds of
// rows once the graph settles, spread over many warps); nch[s] = chunks of s
// Chunks are numbered in the order of `order` (nullable: source ids): position r
// holds source order[r]; nch[r] = chunks of that source.  An order that puts
// nearby points next to each other keeps the rows of the chunks in flight within
// the L2 cache; it changes no result.
__global__ void chunk_count_kernel(const int32_t* __restrict__ off, const int32_t* __restrict__ order, int64_t n,
                                   int32_t* __restrict__ nch) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = order ? order[r] : r;
    nch[r] = (off[s + 1] - off[s] + 15) >> 4;
  }
}

__global__ void chunk_fill_kernel(const int32_t* __restrict__ choff, int64_t n, int32_t* __restrict__ chunk_pos) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
    for (int c = choff[r]; c < choff[r + 1]; ++c) chunk_pos[c] = (int32_t)r;
}

struct JoinArgs {
  const void* Xd;  // float or __half rows of length dd, pitch ldx elements
  const float* sqd;
  int dd, ldx;
  const int32_t* idx_old;
  const int32_t* off;      // n + 1 bucket offsets
  const int32_t* entries;  // i * 32 + p, bucketed by source
  const int32_t* order;    // nullable: source of position r
  const int32_t* choff;    // n + 1 chunk offsets by position (choff[n] = chunks)
  const int32_t* chunk_pos;
  int64_t n;
  int k, mc, j_nn;
  int half_round;
  float* nnbuf;  // (n, mc * j_nn)
  float* curd;   // (n, k), nullable: current-neighbour distances not wanted
  unsigned long long* evals;  // nullable
};

__device__ __forceinline__ int join_col_id(const JoinArgs& a, int64_t s, int col) {
  return col == 0 ? (int)s : a.idx_old[s * a.k + col - 1];
}

__device__ __forceinline__ void join_store(const JoinArgs& a, int64_t s, int ent, int col, float dot) {
  const int64_t i = ent >> 5;
  const int p = ent & 31;
  const int cid = join_col_id(a, s, col);
  const float d = d2_from_dot(a.sqd[i], a.sqd[cid], dot, a.half_round != 0);
  if (col == 0) {
    if (a.curd) a.curd[i * a.k + p] = d;
  } else {
    a.nnbuf[i * (int64_t)(a.mc * a.j_nn) + p * a.j_nn + (col - 1)] = d;
  }
}

// FP16 rows: 16 entries x 16 columns per tile on mma.m16n8k16 (two n-tiles), with
// the k-position map of dists_f16: thread (g, c) loads 16-byte chunk c + 4 st of
// entry rows g, g + 8 and of column rows g, g + 8, so A and B share the map and
// D[m][n] is the full dot product.  D fragments: d0 = columns 2c, 2c + 1 of rows
// g, g + 8; d1 = columns 8 + 2c, 9 + 2c.
// 10 resident blocks per SM (48 registers, a few spilled to L1) rather than the 8 that
// 60 registers allow: more row loads in flight for a kernel bound by them
__global__ void __launch_bounds__(kWarps * 32, 10) join_f16_kernel(JoinArgs a) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t w = (int64_t)blockIdx.x * kWarps + warp;  // chunk
  if (w >= a.choff[a.n]) return;
  const int64_t r = a.chunk_pos[w];
  const int64_t s = a.order ? a.order[r] : r;
  const int beg = a.off[s] + 16 * (int)(w - a.choff[r]);
  const int end = min(a.off[s + 1], beg + 16);
  const int ncol = 1 + a.j_nn;
  const __half* X = reinterpret_cast<const __half*>(a.Xd);
  const int V = a.ldx / 8, S = (V + 3) / 4;
  const int g = lane >> 2, c = lane & 3;
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
  for (int cb = 0; cb < ncol; cb += 16) {
    const bool bv0 = cb + g < ncol, bv1 = cb + g + 8 < ncol;
    const uint4* b0 = reinterpret_cast<const uint4*>(X + (int64_t)(bv0 ? join_col_id(a, s, cb + g) : 0) * a.ldx);
    const uint4* b1 = reinterpret_cast<const uint4*>(X + (int64_t)(bv1 ? join_col_id(a, s, cb + g + 8) : 0) * a.ldx);
    for (int e0 = beg; e0 < end; e0 += 16) {
      const bool av0 = e0 + g < end, av1 = e0 + g + 8 < end;
      const int en0 = av0 ? a.entries[e0 + g] : 0, en1 = av1 ? a.entries[e0 + g + 8] : 0;
      const uint4* r0 = reinterpret_cast<const uint4*>(X + (int64_t)(en0 >> 5) * a.ldx);
      const uint4* r1 = reinterpret_cast<const uint4*>(X + (int64_t)(en1 >> 5) * a.ldx);
      float d0[4] = {0.f, 0.f, 0.f, 0.f}, d1[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 2
      for (int st = 0; st < S; ++st) {
        const int q = c + 4 * st;
        const bool in = q < V;
        const uint4 A0 = (in && av0) ? __ldg(r0 + q) : zero;
        const uint4 A1 = (in && av1) ? __ldg(r1 + q) : zero;
        const uint4 B0 = (in && bv0) ? __ldg(b0 + q) : zero;
        const uint4 B1 = (in && bv1) ? __ldg(b1 + q) : zero;
        mma_f16(d0, A0.x, A1.x, A0.y, A1.y, B0.x, B0.y);
        mma_f16(d0, A0.z, A1.z, A0.w, A1.w, B0.z, B0.w);
        mma_f16(d1, A0.x, A1.x, A0.y, A1.y, B1.x, B1.y);
        mma_f16(d1, A0.z, A1.z, A0.w, A1.w, B1.z, B1.w);
      }
      // this thread's outputs: rows g (en0), g + 8 (en1) x columns cb + {2c, 2c+1, 8+2c, 9+2c}
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const bool rv = h == 0 ? av0 : av1;
        const int en = h == 0 ? en0 : en1;
        if (!rv) continue;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int col = cb + (u < 2 ? 2 * c + u : 8 + 2 * c + (u - 2));
          const float dot = u < 2 ? d0[2 * h + u] : d1[2 * h + (u - 2)];
          if (col < ncol) join_store(a, s, en, col, dot);
        }
      }
    }
  }
  if (lane == 0 && a.evals) {
    const unsigned long long m = (unsigned long long)(end - beg);
    atomicAdd(a.evals, m * (unsigned long long)ncol);
  }
}

// FP32 rows (dd % 4 == 0, 16-byte aligned): 16 entries x 16 columns per tile.  Each
// warp stages its 32 rows (entries 0-15, columns 16-31) slice by slice (32 floats
// of every row) into its own shared memory with cp.async, JS_STAGES slices in
// flight, and computes from there: the two half-warps take alternate float4s of a
// slice, lane m holds entry rows m/4 + {0,4,8,12} x columns m%4 + {0,4,8,12} (eight
// float4 reads feed 64 FMAs), and one shuffle per output adds the halves.  A row
// pitch of 40 floats puts the eight 16-byte reads of each instruction on distinct
// bank groups.
constexpr int JS_STAGES = 2;
constexpr int JS_SLICE = 32;  // floats of each row per stage
constexpr int JS_PITCH = 40;  // floats per staged row
constexpr int JS_WARP_FLOATS = JS_STAGES * 32 * JS_PITCH;

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// 4 resident blocks per SM (at most 128 registers): with two stages the shared memory
// of 4 blocks fits, and the issue-bound kernel wants the warps
__global__ void __launch_bounds__(kWarps * 32, 4) join_f32_kernel(JoinArgs a) {
  extern __shared__ __align__(16) float js_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t w = (int64_t)blockIdx.x * kWarps + warp;  // chunk
  if (w >= a.choff[a.n]) return;
  const int64_t r = a.chunk_pos[w];
  const int64_t s = a.order ? a.order[r] : r;
  const int beg = a.off[s] + 16 * (int)(w - a.choff[r]);
  const int end = min(a.off[s + 1], beg + 16);
  const int ncol = 1 + a.j_nn;
  const float* X = reinterpret_cast<const float*>(a.Xd);
  const int dd = a.dd;
  const int nsl = (dd + JS_SLICE - 1) / JS_SLICE;
  float* buf = js_smem + warp * JS_WARP_FLOATS;
  const uint32_t buf_s = static_cast<uint32_t>(__cvta_generic_to_shared(buf));
  const int half = lane >> 4, m = lane & 15;
  const int at = m >> 2;  // entry rows at + 4u
  const int bt = m & 3;   // columns bt + 4j
  // this lane copies float4 (lane & 7) of staged rows (lane >> 3) + 4v, v = 0..7
  const int f4 = lane & 7;
  for (int cb = 0; cb < ncol; cb += 16) {
    const float* src[8];
    bool vrow[8];
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      const int sr = (lane >> 3) + 4 * v;
      int id = 0;
      if (sr < 16) {
        vrow[v] = beg + sr < end;
        if (vrow[v]) id = a.entries[beg + sr] >> 5;
      } else {
        vrow[v] = cb + sr - 16 < ncol;
        if (vrow[v]) id = join_col_id(a, s, cb + sr - 16);
      }
      src[v] = X + (int64_t)id * a.ldx + f4 * 4;
    }
    auto issue = [&](int sl) {
      if (sl < nsl) {
        const uint32_t stg = buf_s + (uint32_t)((sl % JS_STAGES) * 32 * JS_PITCH * 4);
        const int k0 = sl * JS_SLICE + f4 * 4;
#pragma unroll
        for (int v = 0; v < 8; ++v) {
          const int sr = (lane >> 3) + 4 * v;
          const bool ok = vrow[v] && k0 < dd;  // dd % 4 == 0: a float4 is all in or all out
          cp_async16(stg + (uint32_t)((sr * JS_PITCH + f4 * 4) * 4), ok ? (const void*)(src[v] + sl * JS_SLICE) : X,
                     ok ? 16u : 0u);
        }
      }
      cp_async_commit();
    };
    float acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[u][j] = 0.f;
#pragma unroll
    for (int sl = 0; sl < JS_STAGES - 1; ++sl) issue(sl);
#pragma unroll 1
    for (int sl = 0; sl < nsl; ++sl) {
      cp_async_wait<JS_STAGES - 2>();  // slice sl has landed (this lane's copies)
      __syncwarp();                   // ... and every lane's; slice sl - 1 is consumed
      issue(sl + JS_STAGES - 1);       // into the buffer slice sl - 1 used
      const float* stg = buf + (sl % JS_STAGES) * 32 * JS_PITCH;
#pragma unroll
      for (int jj = 0; jj < JS_SLICE / 8; ++jj) {
        const int c4 = (2 * jj + half) * 4;
        float4 x[4], y[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) x[u] = *reinterpret_cast<const float4*>(stg + (at + 4 * u) * JS_PITCH + c4);
#pragma unroll
        for (int j = 0; j < 4; ++j) y[j] = *reinterpret_cast<const float4*>(stg + (16 + bt + 4 * j) * JS_PITCH + c4);
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            acc[u][j] = fmaf(x[u].x, y[j].x, acc[u][j]);
            acc[u][j] = fmaf(x[u].y, y[j].y, acc[u][j]);
            acc[u][j] = fmaf(x[u].z, y[j].z, acc[u][j]);
            acc[u][j] = fmaf(x[u].w, y[j].w, acc[u][j]);
          }
      }
    }
    cp_async_wait<0>();
    __syncwarp();  // the buffers are free for the next column block
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[u][j] += __shfl_xor_sync(0xffffffffu, acc[u][j], 16);
    if (half == 0) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int e = beg + at + 4 * u;
        if (e >= end) continue;
        const int en = a.entries[e];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int col = cb + bt + 4 * j;
          if (col < ncol) join_store(a, s, en, col, acc[u][j]);
        }
      }
    }
  }
  if (lane == 0 && a.evals) {
    const unsigned long long mm = (unsigned long long)(end - beg);
    atomicAdd(a.evals, mm * (unsigned long long)ncol);
  }
}

// query-row region of a warp: the staged query row (row_bytes), or before it the
// prefetched nn-of-nn distances (pre floats), whichever is larger, 16-byte multiple
__host__ __device__ inline size_t iter_row_region(int row_bytes, int pre) {
  const size_t a = (size_t)row_bytes, b = (size_t)pre * 4;
  return ((a > b ? a : b) + 15) / 16 * 16;
}

// dedup hash (4 hcap bytes), later candidate distances (4 tcap) + to-do list (2 tcap)
__host__ __device__ inline size_t iter_scratch_bytes(int tcap, int hcap) {
  const size_t a = (size_t)hcap * 4, b = (size_t)tcap * 6;
  return ((a > b ? a : b) + 15) / 16 * 16;
}

struct IterArgs {
  const void* Xd;  // distance space, float or __half rows of length dd, pitch ldx elements
  const float* sqd;
  int dd, ldx;
  int group;  // FP32 rows: lanes per candidate (4, 8, 16 or 32)
  const int32_t* idx_old;
  const float* dist_old;
  const uint8_t* flags_old;  // converging path only
  const int32_t* rev;        // nullable
  const int32_t* order;      // nullable: row handled by warp slot r (a locality order)
  const float* nnbuf;        // nullable: nn-of-nn distances from the blocked join
  const float* curd;         // nullable: current-neighbour distances from the join
  int64_t n;
  int k, mc_new, j_nn;
  int converging, recompute_cur, half_round;
  int tcap, hcap, hbits;  // candidate capacity per row (multiple of 32); hash size 2^hbits
  int32_t* idx_new;
  float* dist_new;
  uint8_t* flags_new;
  unsigned long long* changed;
  unsigned long long* evals;  // nullable: distance evaluations performed
};

template <class T>
__global__ void __launch_bounds__(kWarps * 32, 10) iter_kernel(IterArgs a) {
  extern __shared__ __align__(16) uint8_t smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t slot = (int64_t)blockIdx.x * kWarps + warp;
  if (slot >= a.n) return;
  const int64_t row = a.order ? (int64_t)a.order[slot] : slot;
  // per warp: query row (first the prefetched nn-of-nn distances of the join) |
  // candidate ids | scratch (the dedup hash table, then the candidate distances and
  // the to-do list) | sources
  const int nn_cols = a.mc_new * a.j_nn;
  const size_t xs_bytes = iter_row_region(a.ldx * (int)sizeof(T), a.nnbuf ? nn_cols : 0);
  const size_t scratch = iter_scratch_bytes(a.tcap, a.hcap);
  const size_t per_warp = xs_bytes + (size_t)a.tcap * 4 + scratch + 32 * 4;
  uint8_t* base = smem_raw + warp * per_warp;
  T* xs = reinterpret_cast<T*>(base);
  int32_t* cid = reinterpret_cast<int32_t*>(base + xs_bytes);
  uint8_t* scr = reinterpret_cast<uint8_t*>(cid + a.tcap);
  int32_t* htab = reinterpret_cast<int32_t*>(scr);
  float* cd = reinterpret_cast<float*>(scr);
  uint16_t* todo = reinterpret_cast<uint16_t*>(cd + a.tcap);
  int32_t* srcs = reinterpret_cast<int32_t*>(scr + scratch);
  if (row >= a.n) return;
  const int k = a.k;
  const int32_t* orow = a.idx_old + row * k;

  // row-local copy of the old neighbours (lane p holds entry p; k <= 32)
  const int my_old = lane < k ? orow[lane] : -1;
  const float my_old_d = lane < k ? a.dist_old[row * k + lane] : kBig;
  if (a.converging) {
    const bool f = lane < k && a.flags_old[row * k + lane];
    const unsigned fb = __ballot_sync(0xffffffffu, f);
    if (fb == 0) {  // no NEW neighbour: the row keeps its list (nndescent.py:111-126, 211-217)
      if (lane < k) {
        a.idx_new[row * k + lane] = my_old;
        a.dist_new[row * k + lane] = my_old_d;
        a.flags_new[row * k + lane] = 0;
      }
      return;
    }
    // NEW-first stable order (nndescent.py:105-106)
    const unsigned lt = (1u << lane) - 1u;
    const int nnew = __popc(fb);
    const unsigned ob = __ballot_sync(0xffffffffu, lane < k && !f);
    const int pos = f ? __popc(fb & lt) : nnew + __popc(ob & lt);
    if (lane < k) srcs[pos] = my_old;
  } else {
    if (lane < k) srcs[lane] = my_old;
  }
  // the row's nn-of-nn distances from the join, copied into shared memory while
  // the candidate ids and the dedup run (4-byte cp.async: a row starts at any
  // multiple of 4 bytes); phase 3 reads them from there
  float* snn = reinterpret_cast<float*>(base);
  if (a.nnbuf) {
    const float* src = a.nnbuf + row * nn_cols;
    const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(snn));
    for (int t = lane; t < nn_cols; t += 32)
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst + 4u * t), "l"(src + t) : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  for (int t = lane; t < a.hcap; t += 32) htab[t] = -1;
  __syncwarp();

  // 1. candidate ids in the reference's column order
  const int T_total = k + nn_cols + (a.rev ? k : 0);
  // four chunks at a time: their loads are issued together, one round trip
  for (int g0 = 0; g0 < a.tcap; g0 += 128) {
    const int32_t* src_p[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int t = g0 + 32 * u + lane;
      src_p[u] = nullptr;
      if (t < k) {
        src_p[u] = orow + t;
      } else if (t < k + nn_cols) {
        const int q = t - k;
        src_p[u] = a.idx_old + (int64_t)srcs[q / a.j_nn] * k + (q % a.j_nn);
      } else if (t < T_total) {
        src_p[u] = a.rev + row * k + (t - k - nn_cols);
      }
    }
    int v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) v[u] = src_p[u] ? __ldg(src_p[u]) : 0x7fffffff;
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (g0 + 32 * u < a.tcap) cid[g0 + 32 * u + lane] = v[u];
  }
  __syncwarp();

  // 2. first-occurrence dedup (bit c of `keep`: this lane's column in chunk c is the
  // first occurrence of its id and not the row itself)
  unsigned long long keep = 0ull;
  for (int t0 = 0, ch = 0; t0 < a.tcap; t0 += 32, ++ch) {
    const int t = t0 + lane;
    const int id = cid[t];
    const bool valid = t < T_total;
    const unsigned same = __match_any_sync(0xffffffffu, id);
    bool first = valid && (__ffs(same) - 1) == lane;  // lowest lane of an equal-id group in this chunk
    if (first) {
      unsigned h = ((unsigned)id * 0x9E3779B1u) >> (32 - a.hbits);
      while (true) {
        const int old = atomicCAS(&htab[h], -1, id);
        if (old == -1) break;
        if (old == id) {
          first = false;
          break;
        }
        h = (h + 1) & (unsigned)(a.hcap - 1);
      }
    }
    if (first && id != (int)row) keep |= 1ull << ch;
  }
  __syncwarp();  // the hash table is dead; its space becomes cd / todo

  // 3. stored distances and the list of distances to compute
  if (a.nnbuf) {
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncwarp();
  }
  int n_todo = 0;
  for (int t0 = 0, ch = 0; t0 < a.tcap; t0 += 32, ++ch) {
    const int t = t0 + lane;
    float d = kBig;
    bool need = false;
    if ((keep >> ch) & 1ull) {
      if (t < k) {
        if (!a.recompute_cur) d = a.dist_old[row * k + t];
        else if (a.curd && t < a.mc_new) d = a.curd[row * k + t];
        else need = true;
      } else if (a.nnbuf && t < k + nn_cols) {
        d = snn[t - k];
      } else if (a.curd && t >= k + nn_cols) {
        // reverse candidate j: this row sits at some position p of j's list, and
        // for p < mc_new the join computed d(j, row) = d(row, j) as curd[j][p]
        const int64_t j = cid[t];
        const int32_t* jr = a.idx_old + j * k;
        // predicated sweeps of 16 positions (no early exit inside a sweep) keep
        // their loads in flight together; the lowest matching position wins
        int pos = -1;
        for (int q0 = 0; q0 < a.mc_new && pos < 0; q0 += 16) {
#pragma unroll
          for (int u = 15; u >= 0; --u)
            if (q0 + u < a.mc_new && __ldg(jr + q0 + u) == (int)row) pos = q0 + u;
        }
        if (pos >= 0) d = a.curd[j * k + pos];
        else need = true;
      } else {
        need = true;
      }
    }
    cd[t] = d;
    const unsigned nb = __ballot_sync(0xffffffffu, need);
    if (need) todo[n_todo + __popc(nb & ((1u << lane) - 1u))] = (uint16_t)t;
    n_todo += __popc(nb);
  }
  __syncwarp();
  const float sqi = a.sqd[row];
  if (n_todo > 0) {  // the query row, for the distances still to compute
    for (int t = lane; t < a.ldx; t += 32) xs[t] = reinterpret_cast<const T*>(a.Xd)[row * a.ldx + t];
    __syncwarp();
  }
  if constexpr (sizeof(T) == 2) {
    dists_f16(reinterpret_cast<const __half*>(a.Xd), a.ldx, reinterpret_cast<const __half*>(xs), a.sqd, sqi, row,
              cid, todo, n_todo, cd, lane);
  } else if ((a.ldx & 3) == 0 && (a.dd & 3) == 0) {
    dists_f32<true>(reinterpret_cast<const float*>(a.Xd), a.dd, a.ldx, reinterpret_cast<const float*>(xs), a.sqd,
                    sqi, row, cid, todo, n_todo, cd, lane, a.group);
  } else {
    dists_f32<false>(reinterpret_cast<const float*>(a.Xd), a.dd, a.ldx, reinterpret_cast<const float*>(xs), a.sqd,
                     sqi, row, cid, todo, n_todo, cd, lane, a.group);
  }
  __syncwarp();

  // 4. k smallest (distance, id) over all candidate columns.  The list sits one key
  // per lane, ascending, sentinels past k.  Keys of a chunk below the current k-th are
  // inserted one at a time (a ballot, two shuffles); a chunk with more than 10 of them
  // (the first chunk, when the list is empty) is sorted across the warp (bitonic, 15
  // exchange steps) and merged: the 32 smallest of the list and the sorted chunk,
  // paired in reverse, form a bitonic sequence that five exchange steps order.
  constexpr float kSent = kBig * 4.0f;  // above every real key, including 1e30 entries
  float lv = kSent;
  int li = 0x7fffffff;
  float tau = lv;
  int tau_i = li;
  for (int t0 = 0; t0 < a.tcap; t0 += 32) {
    const int t = t0 + lane;
    float d = t < T_total ? cd[t] : kSent;
    int id = t < T_total ? cid[t] : 0x7fffffff;
    unsigned b = __ballot_sync(0xffffffffu, t < T_total && key_lt(d, id, tau, tau_i));
    if (__popc(b) > 10) {
      if (!((b >> lane) & 1u)) {
        d = kSent;
        id = 0x7fffffff;
      }
      warp_sort_keys(d, id, lane);
      const float od = __shfl_sync(0xffffffffu, d, 31 - lane);
      const int oi = __shfl_sync(0xffffffffu, id, 31 - lane);
      if (key_lt(od, oi, lv, li)) {
        lv = od;
        li = oi;
      }
      warp_bitonic_clean(lv, li, lane);
      if (lane >= k) {
        lv = kSent;
        li = 0x7fffffff;
      }
      tau = __shfl_sync(0xffffffffu, lv, k - 1);
      tau_i = __shfl_sync(0xffffffffu, li, k - 1);
      continue;
    }
    while (b) {
      const int src = __ffs(b) - 1;
      const float sd = __shfl_sync(0xffffffffu, d, src);
      const int si = __shfl_sync(0xffffffffu, id, src);
      list_insert(lv, li, sd, si, k, lane);
      tau = __shfl_sync(0xffffffffu, lv, k - 1);
      tau_i = __shfl_sync(0xffffffffu, li, k - 1);
      b &= ~(1u << src);
      b &= __ballot_sync(0xffffffffu, key_lt(d, id, tau, tau_i));
    }
  }
  if (lane < k) {
    a.idx_new[row * k + lane] = li;
    a.dist_new[row * k + lane] = lv;
    const bool ch = li != my_old;
    a.flags_new[row * k + lane] = ch ? 1 : 0;
  }
  const int nch = __popc(__ballot_sync(0xffffffffu, lane < k && li != my_old));
  if (lane == 0 && nch) atomicAdd(a.changed, (unsigned long long)nch);
  if (lane == 0 && a.evals) atomicAdd(a.evals, (unsigned long long)n_todo);
}

}  // namespace nnd
}  // namespace umapb

using namespace umapb;

static size_t iter_smem_per_warp(int ldx, int elem, int tcap, int hcap, int pre) {
  return nnd::iter_row_region(ldx * elem, pre) + (size_t)tcap * 4 + nnd::iter_scratch_bytes(tcap, hcap) + 32 * 4;
}

namespace umapb {
namespace nnd {
__global__ void sqrt_kernel(const float* __restrict__ d2, int64_t m, float* __restrict__ out) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x)
    out[t] = sqrtf(fmaxf(d2[t], 0.0f));
}
}  // namespace nnd
}  // namespace umapb

extern "C" int umapb_nnd_sqrt(const float* d2, int64_t count, float* out, umapb_stream_t stream_) {
  clear_error();
  UMAPB_REQUIRE(d2 && out && count >= 0, "nnd_sqrt: bad arguments");
  if (count == 0) return UMAPB_OK;
  const int64_t want = ceil_div(count, 256);
  const unsigned blocks = (unsigned)(want < num_sms() * 8 ? want : num_sms() * 8);
  nnd::sqrt_kernel<<<blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream_)>>>(d2, count, out);
  UMAPB_LAUNCH_CHECK("nnd_sqrt kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_nnd_sqnorms(const void* X, int64_t n, int32_t dd, int32_t half, float* sq,
                                 umapb_stream_t stream_) {
  clear_error();
  UMAPB_REQUIRE(X && sq && n >= 1 && dd >= 1, "nnd_sqnorms: bad arguments");
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  const unsigned blocks = (unsigned)ceil_div(n * 32, 256);
  if (half)
    nnd::sqnorm_kernel<__half><<<blocks, 256, 0, stream>>>(static_cast<const __half*>(X), n, dd, sq);
  else
    nnd::sqnorm_kernel<float><<<blocks, 256, 0, stream>>>(static_cast<const float*>(X), n, dd, sq);
  UMAPB_LAUNCH_CHECK("nnd_sqnorms kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_nnd_to_half(const float* X, int64_t n, int32_t dd, int32_t ldh, void* H,
                                 umapb_stream_t stream_) {
  clear_error();
  UMAPB_REQUIRE(X && H && n >= 0 && dd >= 1 && ldh >= dd, "nnd_to_half: bad arguments");
  const int64_t count = n * ldh;
  if (count == 0) return UMAPB_OK;
  const int64_t want = ceil_div(count, 256);
  const unsigned blocks = (unsigned)(want < num_sms() * 8 ? want : num_sms() * 8);
  nnd::to_half_kernel<<<blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream_)>>>(X, n, dd, ldh,
                                                                                    static_cast<__half*>(H));
  UMAPB_LAUNCH_CHECK("nnd_to_half kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_nnd_gather(const float* X, const float* sq, int64_t n, int32_t dd, int32_t* idx, float* dist,
                                int32_t k, int32_t sort_rows, umapb_stream_t stream_) {
  clear_error();
  UMAPB_REQUIRE(X && sq && idx && dist, "nnd_gather: null array argument");
  UMAPB_REQUIRE(n >= 1 && dd >= 1 && k >= 1 && k <= nnd_wide_max_k(), "nnd_gather: need 1 <= k <= %d",
                nnd_wide_max_k());
  if (k > 32)
    return nnd_gather_wide(X, sq, n, dd, idx, dist, k, sort_rows, reinterpret_cast<cudaStream_t>(stream_));
  const size_t smem = (size_t)nnd::kWarps * dd * sizeof(float);
  UMAPB_REQUIRE(smem <= 200 * 1024, "nnd_gather: row dimension too large");
  {
    static std::mutex mu;
    static bool attr[64] = {false};
    int dev = 0;
    UMAPB_CUDA_TRY(cudaGetDevice(&dev), "nnd_gather: device");
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < 64 && !attr[dev]) {
      UMAPB_CUDA_TRY(cudaFuncSetAttribute(nnd::gather_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          200 * 1024),
                     "nnd_gather: smem attribute");
      attr[dev] = true;
    }
  }
  nnd::gather_rows_kernel<<<(unsigned)ceil_div(n, nnd::kWarps), nnd::kWarps * 32, smem,
                            reinterpret_cast<cudaStream_t>(stream_)>>>(X, sq, n, dd, idx, dist, k, sort_rows);
  UMAPB_LAUNCH_CHECK("nnd_gather kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_nnd_gather_pairs(const float* X, const float* sq, int64_t n, int32_t dd, const int32_t* idx,
                                      float* dist, int32_t k, int64_t r0, int64_t r1, umapb_stream_t stream_) {
  clear_error();
  UMAPB_REQUIRE(X && sq && idx && dist, "nnd_gather_pairs: null array argument");
  UMAPB_REQUIRE(n >= 1 && dd >= 1 && k >= 1 && k <= 32, "nnd_gather_pairs: need n >= 1, dd >= 1, 1 <= k <= 32");
  UMAPB_REQUIRE(0 <= r0 && r0 <= r1 && r1 <= n, "nnd_gather_pairs: need 0 <= r0 <= r1 <= n");
  const size_t smem = (size_t)nnd::kWarps * dd * sizeof(float);
  UMAPB_REQUIRE(smem <= 200 * 1024, "nnd_gather_pairs: row dimension too large");
  if (r1 == r0) return UMAPB_OK;
  {
    static std::mutex mu;
    static bool attr[64] = {false};
    int dev = 0;
    UMAPB_CUDA_TRY(cudaGetDevice(&dev), "nnd_gather_pairs: device");
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < 64 && !attr[dev]) {
      UMAPB_CUDA_TRY(cudaFuncSetAttribute(nnd::gather_pairs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          200 * 1024),
                     "nnd_gather_pairs: smem attribute");
      attr[dev] = true;
    }
  }
  nnd::gather_pairs_kernel<<<(unsigned)ceil_div(r1, nnd::kWarps), nnd::kWarps * 32, smem,
                             reinterpret_cast<cudaStream_t>(stream_)>>>(X, sq, dd, idx, dist, k, r0, r1);
  UMAPB_LAUNCH_CHECK("nnd_gather_pairs kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_nnd_sort_rows(int32_t* idx, float* dist, int64_t n, int32_t k, umapb_stream_t stream_) {
  clear_error();
  UMAPB_REQUIRE(idx && dist, "nnd_sort_rows: null array argument");
  UMAPB_REQUIRE(n >= 1 && k >= 1 && k <= 32, "nnd_sort_rows: need n >= 1 and 1 <= k <= 32");
  nnd::sort_rows_kernel<<<(unsigned)ceil_div(n, nnd::kWarps), nnd::kWarps * 32, 0,
                          reinterpret_cast<cudaStream_t>(stream_)>>>(idx, dist, n, k);
  UMAPB_LAUNCH_CHECK("nnd_sort_rows kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_nnd_reverse_workspace(int64_t n, int32_t k, size_t* bytes) {
  clear_error();
  UMAPB_REQUIRE(bytes && n >= 1 && k >= 1, "nnd_reverse_workspace: bad arguments");
  Carver c(nullptr);
  c.take<int32_t>(64);
  c.take<int32_t>((size_t)n + 1);  // degree -> offsets
  c.take<int32_t>((size_t)n + 1);  // fill counters
  c.take<int32_t>((size_t)n);      // degree copy
  c.take<int32_t>((size_t)n * k);  // buckets
  c.take<int64_t>(8 + kScanMaxBlocks);  // totals, then scan_exclusive's block totals
  *bytes = c.bytes();
  return UMAPB_OK;
}

extern "C" int umapb_nnd_reverse(const int32_t* idx, int64_t n, int32_t k, int32_t* rev, void* workspace,
                                 size_t workspace_bytes, umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(idx && rev && n >= 1 && k >= 1, "nnd_reverse: bad arguments");
  UMAPB_REQUIRE(n < ((int64_t)1 << 31) / 2, "nnd_reverse: n too large");
  Carver c(workspace);
  c.take<int32_t>(64);
  int32_t* off = c.take<int32_t>((size_t)n + 1);
  int32_t* fill = c.take<int32_t>((size_t)n + 1);
  int32_t* deg = c.take<int32_t>((size_t)n);
  int32_t* bucket = c.take<int32_t>((size_t)n * k);
  int64_t* total = c.take<int64_t>(8 + kScanMaxBlocks);  // total, then scan scratch at total + 8
  if (!workspace || workspace_bytes < c.bytes())
    return set_error(UMAPB_ERR_WORKSPACE, "nnd_reverse: workspace of %zu bytes, need %zu", workspace_bytes, c.bytes());
  const int64_t m = n * k;
  UMAPB_CUDA_TRY(cudaMemsetAsync(off, 0, sizeof(int32_t) * (n + 1), stream), "nnd_reverse: reset");
  UMAPB_CUDA_TRY(cudaMemsetAsync(fill, 0, sizeof(int32_t) * (n + 1), stream), "nnd_reverse: reset");
  const int64_t want = ceil_div(m, 256);
  const unsigned blocks = (unsigned)(want < num_sms() * 8 ? want : num_sms() * 8);
  nnd::indegree_kernel<<<blocks, 256, 0, stream>>>(idx, m, off);
  UMAPB_CUDA_TRY(cudaMemcpyAsync(deg, off, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, stream),
                 "nnd_reverse: degree copy");
  scan_exclusive(off, n, total, total + 8, stream);
  nnd::bucket_fill_kernel<<<blocks, 256, 0, stream>>>(idx, m, k, off, fill, bucket);
  nnd::bucket_select_kernel<<<(unsigned)ceil_div(n, nnd::kWarps * nnd::kSelRows), nnd::kWarps * 32, 0, stream>>>(
      bucket, off, deg, n, k, 0, rev);
  UMAPB_LAUNCH_CHECK("nnd_reverse kernels");
  count_launches(4);
  return UMAPB_OK;
}

extern "C" int umapb_nnd_join_workspace(int64_t n, int32_t k, int32_t mc, size_t* bytes) {
  clear_error();
  UMAPB_REQUIRE(bytes && n >= 1 && k >= 1 && mc >= 0 && mc <= k, "nnd_join_workspace: bad arguments");
  Carver c(nullptr);
  c.take<int32_t>(64);
  c.take<int32_t>((size_t)n + 1);                // source counts -> bucket offsets
  c.take<int32_t>((size_t)n + 1);                // fill counters
  c.take<int32_t>((size_t)n * (mc > 0 ? mc : 1));  // entries
  c.take<int32_t>((size_t)n + 1);                // chunk counts -> chunk offsets
  c.take<int32_t>((size_t)n + (size_t)n * mc / 16 + 1);  // chunk -> source
  c.take<int64_t>(8 + kScanMaxBlocks);  // totals, then scan_exclusive's block totals
  c.take<int32_t>((size_t)n * (mc > 0 ? mc : 1));  // the NEW-first source lists (umapb_nnd_join_new)
  *bytes = c.bytes();
  return UMAPB_OK;
}

// The blocked join over the sources idx_old[i][p < mc] or, with flags, over the
// NEW-first source lists of the converging path (new_sources_kernel).
static int join_impl(const void* Xd, const float* sqd, int32_t dd, int32_t ldx, int32_t half,
                     const int32_t* idx_old, const uint8_t* flags, const int32_t* order, int64_t n, int32_t k,
                     int32_t mc, int32_t j_nn, float* nnbuf, float* curd, int32_t* rev_out,
                     unsigned long long* evals, void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  UMAPB_REQUIRE(Xd && sqd && idx_old, "nnd_join: null array argument");
  UMAPB_REQUIRE(n >= 2 && dd >= 1 && ldx >= dd, "nnd_join: bad shape");
  UMAPB_REQUIRE(n < ((int64_t)1 << 26), "nnd_join: n must be below 2^26");
  UMAPB_REQUIRE(k >= 1 && k <= 32, "nnd_join: k must be in [1, 32]");
  UMAPB_REQUIRE(mc >= 0 && mc <= k && j_nn >= 0 && j_nn <= k, "nnd_join: bad mc / j_nn");
  UMAPB_REQUIRE(!(mc > 0 && j_nn > 0) || nnbuf, "nnd_join: nnbuf is null");
  UMAPB_REQUIRE(!rev_out || mc == k, "nnd_join: reverse candidates from the join need mc == k");
  if (half)
    UMAPB_REQUIRE(ldx % 8 == 0 && (reinterpret_cast<uintptr_t>(Xd) & 15) == 0,
                  "nnd_join: FP16 rows need a pitch that is a multiple of 8 and a 16-byte aligned base");
  else
    UMAPB_REQUIRE(dd % 4 == 0 && ldx % 4 == 0 && (reinterpret_cast<uintptr_t>(Xd) & 15) == 0,
                  "nnd_join: FP32 rows need dd and the pitch multiples of 4 and a 16-byte aligned base");
  Carver c(workspace);
  c.take<int32_t>(64);
  int32_t* off = c.take<int32_t>((size_t)n + 1);
  int32_t* fill = c.take<int32_t>((size_t)n + 1);
  int32_t* entries = c.take<int32_t>((size_t)n * (mc > 0 ? mc : 1));
  int32_t* choff = c.take<int32_t>((size_t)n + 1);
  const int64_t max_chunks = n + n * mc / 16;  // sum of ceil(count / 16) <= n + n*mc/16
  int32_t* chunk_pos = c.take<int32_t>((size_t)max_chunks + 1);
  int64_t* total = c.take<int64_t>(8 + kScanMaxBlocks);  // total, then scan scratch at total + 8
  int32_t* srcs = c.take<int32_t>((size_t)n * (mc > 0 ? mc : 1));
  if (!workspace || workspace_bytes < c.bytes())
    return set_error(UMAPB_ERR_WORKSPACE, "nnd_join: workspace of %zu bytes, need %zu", workspace_bytes, c.bytes());
  if (mc == 0) return UMAPB_OK;
  const int64_t m = n * mc;
  UMAPB_CUDA_TRY(cudaMemsetAsync(off, 0, sizeof(int32_t) * (n + 1), stream), "nnd_join: reset");
  UMAPB_CUDA_TRY(cudaMemsetAsync(fill, 0, sizeof(int32_t) * (n + 1), stream), "nnd_join: reset");
  const int64_t want = ceil_div(m, 256);
  const unsigned blocks = (unsigned)(want < num_sms() * 8 ? want : num_sms() * 8);
  if (flags)
    nnd::new_sources_kernel<<<(unsigned)ceil_div(n * 32, 256), 256, 0, stream>>>(idx_old, flags, n, k, mc, srcs);
  else
    srcs = nullptr;
  nnd::src_count_kernel<<<blocks, 256, 0, stream>>>(idx_old, srcs, n, k, mc, off);
  scan_exclusive(off, n + 1, total, total + 8, stream);
  nnd::src_fill_kernel<<<blocks, 256, 0, stream>>>(idx_old, srcs, n, k, mc, off, fill, entries);
  if (rev_out) {  // with mc == k the buckets are the reverse-candidate buckets
    nnd::bucket_select_kernel<<<(unsigned)ceil_div(n, nnd::kWarps * nnd::kSelRows), nnd::kWarps * 32, 0,
                                stream>>>(entries, off, nullptr, n, k, 5, rev_out);
  }
  const unsigned sblocks = (unsigned)ceil_div(n, 256);
  UMAPB_CUDA_TRY(cudaMemsetAsync(choff + n, 0, sizeof(int32_t), stream), "nnd_join: reset");
  nnd::chunk_count_kernel<<<sblocks, 256, 0, stream>>>(off, order, n, choff);
  scan_exclusive(choff, n + 1, total, total + 8, stream);
  nnd::chunk_fill_kernel<<<sblocks, 256, 0, stream>>>(choff, n, chunk_pos);
  nnd::JoinArgs a;
  a.Xd = Xd;
  a.sqd = sqd;
  a.dd = dd;
  a.ldx = ldx;
  a.idx_old = idx_old;
  a.off = off;
  a.entries = entries;
  a.order = order;
  a.choff = choff;
  a.chunk_pos = chunk_pos;
  a.n = n;
  a.k = k;
  a.mc = mc;
  a.j_nn = j_nn;
  a.half_round = half;
  a.nnbuf = nnbuf;
  a.curd = curd;
  a.evals = evals;
  const unsigned jb = (unsigned)ceil_div(max_chunks, nnd::kWarps);  // warps past the chunk count exit
  if (half) {
    nnd::join_f16_kernel<<<jb, nnd::kWarps * 32, 0, stream>>>(a);
  } else {
    const size_t jsmem = (size_t)nnd::kWarps * nnd::JS_WARP_FLOATS * sizeof(float);
    static std::mutex mu;
    static bool js_attr[64] = {false};
    int dev = 0;
    UMAPB_CUDA_TRY(cudaGetDevice(&dev), "nnd_join: device");
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 0 || dev >= 64 || !js_attr[dev]) {
      UMAPB_CUDA_TRY(cudaFuncSetAttribute(nnd::join_f32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)jsmem),
                     "nnd_join: smem attribute");
      if (dev >= 0 && dev < 64) js_attr[dev] = true;
    }
    nnd::join_f32_kernel<<<jb, nnd::kWarps * 32, jsmem, stream>>>(a);
  }
  UMAPB_LAUNCH_CHECK("nnd_join kernels");
  count_launches((rev_out ? 8 : 7) + (flags ? 1 : 0));
  return UMAPB_OK;
}

extern "C" int umapb_nnd_join(const void* Xd, const float* sqd, int32_t dd, int32_t ldx, int32_t half,
                              const int32_t* idx_old, const int32_t* order, int64_t n, int32_t k, int32_t mc,
                              int32_t j_nn, float* nnbuf,
                              float* curd, int32_t* rev_out, unsigned long long* evals, void* workspace,
                              size_t workspace_bytes, umapb_stream_t stream_) {
  clear_error();
  return join_impl(Xd, sqd, dd, ldx, half, idx_old, nullptr, order, n, k, mc, j_nn, nnbuf, curd, rev_out, evals,
                   workspace, workspace_bytes, reinterpret_cast<cudaStream_t>(stream_));
}

extern "C" int umapb_nnd_join_new(const float* X, const float* sq, int32_t dd, const int32_t* idx_old,
                                  const uint8_t* flags_old, const int32_t* order, int64_t n, int32_t k, int32_t mc,
                                  int32_t j_nn, float* nnbuf, unsigned long long* evals, void* workspace,
                                  size_t workspace_bytes, umapb_stream_t stream_) {
  clear_error();
  UMAPB_REQUIRE(flags_old, "nnd_join_new: null flags");
  return join_impl(X, sq, dd, dd, 0, idx_old, flags_old, order, n, k, mc, j_nn, nnbuf, nullptr, nullptr, evals,
                   workspace, workspace_bytes, reinterpret_cast<cudaStream_t>(stream_));
}

extern "C" int umapb_nnd_iteration(const void* Xd, const float* sqd, int32_t dd, int32_t ldx, int32_t half,
                                   const int32_t* idx_old,
                                   const float* dist_old, const uint8_t* flags_old, const int32_t* rev,
                                   const int32_t* order, const float* nnbuf, const float* curd, int64_t n,
                                   int32_t k, int32_t mc_new, int32_t j_nn, int32_t converging,
                                   int32_t recompute_cur, int32_t* idx_new, float* dist_new, uint8_t* flags_new,
                                   unsigned long long* changed, unsigned long long* evals,
                                   umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(Xd && sqd && idx_old && dist_old && idx_new && dist_new && flags_new && changed,
                "nnd_iteration: null array argument");
  UMAPB_REQUIRE(!converging || flags_old, "nnd_iteration: the converging path needs the flags");
  UMAPB_REQUIRE(n >= 2 && dd >= 1 && ldx >= dd, "nnd_iteration: bad shape");
  UMAPB_REQUIRE(!half || (ldx % 8 == 0 && (reinterpret_cast<uintptr_t>(Xd) & 15) == 0),
                "nnd_iteration: FP16 rows need a pitch that is a multiple of 8 and a 16-byte aligned base");
  UMAPB_REQUIRE(half || ldx % 4 != 0 || dd % 4 != 0 || (reinterpret_cast<uintptr_t>(Xd) & 15) == 0,
                "nnd_iteration: FP32 rows need a 16-byte aligned base");
  UMAPB_REQUIRE(k >= 1 && k <= nnd_wide_max_k(), "nnd_iteration: k must be in [1, %d]", nnd_wide_max_k());
  UMAPB_REQUIRE(mc_new >= 0 && mc_new <= k && j_nn >= 0 && j_nn <= k, "nnd_iteration: bad mc_new / j_nn");
  if (k > 32) {  // one block per row; every candidate distance computed in the row kernel
    UMAPB_REQUIRE(!nnbuf && !curd, "nnd_iteration: the blocked join serves k <= 32 only");
    return nnd_iteration_wide(Xd, sqd, dd, ldx, half, idx_old, dist_old, flags_old, rev, n, k, mc_new, j_nn,
                              converging, recompute_cur, idx_new, dist_new, flags_new, changed, evals, stream);
  }
  nnd::IterArgs a;
  a.Xd = Xd;
  a.sqd = sqd;
  a.dd = dd;
  a.ldx = ldx;
  {
    const int V = half ? ldx / 8 : (ldx + 3) / 4;  // 16-byte chunks per row
    a.group = V <= 32 ? 4 : V <= 128 ? 8 : 16;
  }
  a.idx_old = idx_old;
  a.dist_old = dist_old;
  a.flags_old = flags_old;
  a.rev = rev;
  a.order = order;
  a.nnbuf = nnbuf;  // the converging path's comes from umapb_nnd_join_new
  a.curd = converging ? nullptr : curd;
  a.n = n;
  a.k = k;
  a.mc_new = mc_new;
  a.j_nn = j_nn;
  a.converging = converging;
  a.recompute_cur = recompute_cur;
  a.half_round = half;
  const int T = k + mc_new * j_nn + (rev ? k : 0);
  a.tcap = (T + 31) / 32 * 32;
  int h = 64, hb = 6;
  while (h < 2 * T) {
    h <<= 1;
    ++hb;
  }
  a.hcap = h;
  a.hbits = hb;
  a.idx_new = idx_new;
  a.dist_new = dist_new;
  a.flags_new = flags_new;
  a.changed = changed;
  a.evals = evals;
  const size_t smem = (size_t)nnd::kWarps *
                      iter_smem_per_warp(ldx, half ? 2 : 4, a.tcap, a.hcap, a.nnbuf ? mc_new * j_nn : 0);
  UMAPB_REQUIRE(smem <= 200 * 1024, "nnd_iteration: row dimension too large for shared memory");
  {
    static std::mutex mu;
    static bool attr[64] = {false};
    int dev = 0;
    UMAPB_CUDA_TRY(cudaGetDevice(&dev), "nnd_iteration: device");
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < 64 && !attr[dev]) {
      UMAPB_CUDA_TRY(cudaFuncSetAttribute(nnd::iter_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          200 * 1024),
                     "nnd_iteration: smem attribute");
      UMAPB_CUDA_TRY(cudaFuncSetAttribute(nnd::iter_kernel<__half>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          200 * 1024),
                     "nnd_iteration: smem attribute");
      attr[dev] = true;
    }
  }
  const unsigned blocks = (unsigned)ceil_div(n, nnd::kWarps);
  if (half)
    nnd::iter_kernel<__half><<<blocks, nnd::kWarps * 32, smem, stream>>>(a);
  else
    nnd::iter_kernel<float><<<blocks, nnd::kWarps * 32, smem, stream>>>(a);
  UMAPB_LAUNCH_CHECK("nnd_iteration kernel");
  count_launches(1);
  return UMAPB_OK;
}
