// Spectral initialisation — replaces UMAP._spectral_init, mlx_vis/_umap/umap.py:298-348.
//
// The reference: degrees by scatter-add (float32, edge order), d^-1/2, normalised
// weights w * d_r^-1/2 * d_c^-1/2, then 100 x { V = W V (gather + scatter-add);
// modified Gram-Schmidt with norm sqrt(|v|^2 + 1e-10) } on V (n x (c+1)), take
// columns 1..c, scale by 10 / max|e|, add N(0, 1e-4) noise (NumPy, host) and
// min-max each column to [0, 10].
//
// Here the edges are in row-major order, so W V is a CSR SpMV without atomics
// (2 lanes per row, FP64 partial sums combined by shuffles; V kept in FP32 rows
// padded to 16 bytes, one vector load per edge, Gram matrix and R^-1 in FP64).  MGS of the
// (c+1)-column block equals Q = V R^-1 with R the Cholesky factor of the Gram
// matrix V^T V (+1e-10 on each pivot, as in the reference's norms), so each
// iteration is ONE kernel: it applies the previous iteration's R^-1 to every
// gathered row on the fly and accumulates the new Gram matrix in FP64; its last
// block factors that Gram matrix for the next iteration.
#include <math.h>
#include <stdlib.h>

#include "common.cuh"
#include "philox.cuh"

namespace umapb {
namespace spectral {

constexpr int kBlock = 256;
constexpr int kMaxCols = 5;   // the fused kernels: n_components <= 4
constexpr int kLanes = 2;     // lanes per row in the power iteration
constexpr int kWideCols = 33; // the warp-per-row kernels: n_components <= 32
constexpr int kWideRows = 32; // rows per block in the warp-per-row SpMV

__global__ void row_ptr_kernel(const int32_t* __restrict__ rows, const int64_t* __restrict__ n_edges, int64_t n,
                               int64_t* __restrict__ row_ptr) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r > n) return;
  const int64_t E = *n_edges;
  int64_t lo = 0, hi = E;  // lower_bound of r in rows[0, E)
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (rows[mid] < r) lo = mid + 1;
    else hi = mid;
  }
  row_ptr[r] = lo;
}

// degree (float32, reference edge order), then normalised weights
__global__ void degree_kernel(const float* __restrict__ vals, const int64_t* __restrict__ row_ptr, int64_t n,
                              float* __restrict__ dis) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  float d = 0.f;
  for (int64_t e = row_ptr[r]; e < row_ptr[r + 1]; ++e) d = __fadd_rn(d, vals[e]);
  d = fmaxf(d, 1e-10f);
  dis[r] = __fdiv_rn(1.0f, sqrtf(d));
}

__global__ void norm_weight_kernel(const int32_t* __restrict__ rows, const int32_t* __restrict__ cols,
                                   const float* __restrict__ vals, const int64_t* __restrict__ n_edges,
                                   const float* __restrict__ dis, float* __restrict__ wn) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= *n_edges) return;
  wn[e] = __fmul_rn(__fmul_rn(vals[e], dis[rows[e]]), dis[cols[e]]);
}

// R (upper triangular) from the Gram matrix G with pivots sqrt(g - sum r^2 + 1e-10);
// returns Rinv (upper triangular) in `ri`.  kk <= kMaxCols.
__device__ void chol_inverse(const double* G, int kk, double* ri) {
  double R[kMaxCols][kMaxCols];
  for (int j = 0; j < kk; ++j) {
    for (int i = 0; i < j; ++i) {
      double s = G[i * kk + j];
      for (int p = 0; p < i; ++p) s -= R[p][i] * R[p][j];
      R[i][j] = s / R[i][i];
    }
    double s = G[j * kk + j];
    for (int p = 0; p < j; ++p) s -= R[p][j] * R[p][j];
    R[j][j] = sqrt(fmax(s, 0.0) + 1e-10);
    for (int i = j + 1; i < kk; ++i) R[i][j] = 0.0;
  }
  // invert the upper-triangular R column by column
  for (int j = 0; j < kk; ++j) {
    for (int i = kk - 1; i >= 0; --i) {
      double s = (i == j) ? 1.0 : 0.0;
      for (int p = i + 1; p < kk; ++p) s -= R[i][p] * ri[p * kk + j];
      ri[i * kk + j] = (i <= j) ? s / R[i][i] : 0.0;
    }
  }
}

// One power iteration: Vout = W (Vin Rinv_in); G_out += Vout^T Vout.  Rinv_in ==
// nullptr means the identity (the first multiplication uses V0 as is).  kLanes
// lanes per row stride over its edges (rows of the symmetrised graph range from a
// few edges to hundreds) and meet by shuffles.  The last block to finish (a counter
// per iteration) factors the completed G_out once and writes Rinv_out for the next
// iteration.
__global__ void spmv_gram_kernel(const float* __restrict__ Vin, const double* __restrict__ Rinv_in,
                                 const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ cols,
                                 const float* __restrict__ wn, int64_t n, int kk, int vp, float* __restrict__ Vout,
                                 double* __restrict__ G_out, unsigned* __restrict__ counter,
                                 double* __restrict__ Rinv_out) {
  __shared__ double ri[kMaxCols * kMaxCols];
  __shared__ double gsum[kBlock / 32][kMaxCols * kMaxCols];
  __shared__ bool last;
  if (threadIdx.x < kk * kk)
    ri[threadIdx.x] = Rinv_in ? Rinv_in[threadIdx.x] : ((threadIdx.x % (kk + 1) == 0) ? 1.0 : 0.0);
  __syncthreads();
  const int sub = threadIdx.x & (kLanes - 1);
  const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / kLanes;
  double acc[kMaxCols] = {0, 0, 0, 0, 0};
  if (r < n) {
    const int64_t e1 = row_ptr[r + 1];
    for (int64_t e = row_ptr[r] + sub; e < e1; e += kLanes) {
      const int64_t c = cols[e];
      const double w = (double)wn[e];
      double v[kMaxCols];
      const float4 a = reinterpret_cast<const float4*>(Vin + c * vp)[0];  // rows padded to 4 or 8 floats
      v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w;
      if (kk > 4) v[4] = Vin[c * vp + 4];
      for (int j = 0; j < kk; ++j) {  // q_j = sum_i v_i Rinv[i][j]
        double q = 0.0;
        for (int i = 0; i <= j; ++i) q += v[i] * ri[i * kk + j];
        acc[j] += w * q;
      }
    }
  }
  for (int j = 0; j < kk; ++j) {
#pragma unroll
    for (int o = kLanes / 2; o > 0; o >>= 1) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], o);
  }
  if (r < n && sub == 0)
    for (int j = 0; j < vp; ++j) Vout[r * vp + j] = j < kk ? (float)acc[j] : 0.f;
  if (sub != 0)
    for (int j = 0; j < kk; ++j) acc[j] = 0.0;  // one copy of each row in the Gram sum
  // block reduction of the Gram matrix
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = 0; i < kk; ++i) {
    for (int j = i; j < kk; ++j) {
      double g = acc[i] * acc[j];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
      if (lane == 0) gsum[warp][i * kk + j] = g;
    }
  }
  __syncthreads();
  if (threadIdx.x < kk * kk) {
    const int i = threadIdx.x / kk, j = threadIdx.x % kk;
    if (i <= j) {
      double g = 0.0;
      for (int w = 0; w < kBlock / 32; ++w) g += gsum[w][i * kk + j];
      atomicAdd(&G_out[i * kk + j], g);
      if (i != j) atomicAdd(&G_out[j * kk + i], g);
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    double G[kMaxCols * kMaxCols];
    for (int i = 0; i < kk * kk; ++i) G[i] = __ldcg(G_out + i);
    chol_inverse(G, kk, Rinv_out);
  }
}


// ---- n_components 5..32: one warp per row, lane j holds column j (and j + 32) ----
// Cholesky factor R of the kk x kk Gram matrix (pivots sqrt(g - sum r^2 + 1e-10),
// the same expressions and summation order as chol_inverse) and its inverse, by the
// whole block in shared memory.  g is overwritten with R (upper triangle).
__device__ void chol_inverse_block(double* g, int kk, double* ri) {
  for (int i = 0; i < kk; ++i) {
    if (threadIdx.x == 0) {
      double s = g[i * kk + i];
      for (int p = 0; p < i; ++p) s -= g[p * kk + i] * g[p * kk + i];
      g[i * kk + i] = sqrt(fmax(s, 0.0) + 1e-10);
    }
    __syncthreads();
    for (int j = i + 1 + threadIdx.x; j < kk; j += blockDim.x) {
      double s = g[i * kk + j];
      for (int p = 0; p < i; ++p) s -= g[p * kk + i] * g[p * kk + j];
      g[i * kk + j] = s / g[i * kk + i];
    }
    __syncthreads();
  }
  for (int j = threadIdx.x; j < kk; j += blockDim.x) {  // column j of R^-1
    for (int i = kk - 1; i >= 0; --i) {
      double s = (i == j) ? 1.0 : 0.0;
      for (int p = i + 1; p < kk; ++p) s -= (p > j ? 0.0 : g[i * kk + p] * ri[p * kk + j]);
      ri[i * kk + j] = (i <= j) ? s / g[i * kk + i] : 0.0;
    }
  }
  __syncthreads();
}

// q_j = sum_{i <= j} u_i Rinv[i][j] for the columns j = lane and lane + 32 of a warp's row
__device__ __forceinline__ void apply_rinv_wide(double u0, double u1, const double* ri, int kk, int lane,
                                                double& q0, double& q1) {
  q0 = 0.0, q1 = 0.0;
  for (int i = 0; i < kk; ++i) {
    const double ui = __shfl_sync(0xffffffffu, i < 32 ? u0 : u1, i & 31);
    if (lane < kk && i <= lane) q0 += ui * ri[i * kk + lane];
    if (lane + 32 < kk && i <= lane + 32) q1 += ui * ri[i * kk + lane + 32];
  }
}

// One power iteration for kk > kMaxCols: Vout = (W Vin) Rinv_in (W Vin in FP64 per
// row, one warp per row), G_out += Vout^T Vout from the block's rows staged in
// shared memory; the last block factors G_out into Rinv_out.
__global__ void __launch_bounds__(kBlock) spmv_gram_wide_kernel(
    const float* __restrict__ Vin, const double* __restrict__ Rinv_in, const int64_t* __restrict__ row_ptr,
    const int32_t* __restrict__ cols, const float* __restrict__ wn, int64_t n, int kk, int vp,
    float* __restrict__ Vout, double* __restrict__ G_out, unsigned* __restrict__ counter,
    double* __restrict__ Rinv_out) {
  __shared__ double ri[kWideCols * kWideCols];
  __shared__ double gl[kWideCols * kWideCols];
  __shared__ double vs[kWideRows][kWideCols];
  __shared__ bool last;
  for (int t = threadIdx.x; t < kk * kk; t += blockDim.x)
    ri[t] = Rinv_in ? Rinv_in[t] : ((t % (kk + 1) == 0) ? 1.0 : 0.0);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t rb = (int64_t)blockIdx.x * kWideRows;
  for (int lr = warp; lr < kWideRows; lr += kBlock / 32) {
    const int64_t r = rb + lr;
    double u0 = 0.0, u1 = 0.0;
    if (r < n) {
      const int64_t e1 = row_ptr[r + 1];
      for (int64_t e = row_ptr[r]; e < e1; ++e) {
        const int64_t c = cols[e];
        const double w = (double)wn[e];
        if (lane < kk) u0 += w * (double)Vin[c * vp + lane];
        if (lane + 32 < kk) u1 += w * (double)Vin[c * vp + lane + 32];
      }
    }
    double q0, q1;
    apply_rinv_wide(u0, u1, ri, kk, lane, q0, q1);
    if (r < n) {
      if (lane < vp) Vout[r * vp + lane] = lane < kk ? (float)q0 : 0.f;
      if (lane + 32 < vp) Vout[r * vp + lane + 32] = lane + 32 < kk ? (float)q1 : 0.f;
    }
    vs[lr][lane] = (r < n && lane < kk) ? q0 : 0.0;
    if (lane + 32 < kWideCols) vs[lr][lane + 32] = (r < n && lane + 32 < kk) ? q1 : 0.0;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < kk * kk; t += blockDim.x) {
    const int i = t / kk, j = t % kk;
    if (i <= j) {
      double g = 0.0;
      for (int lr = 0; lr < kWideRows; ++lr) g += vs[lr][i] * vs[lr][j];
      atomicAdd(&G_out[i * kk + j], g);
      if (i != j) atomicAdd(&G_out[j * kk + i], g);
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int t = threadIdx.x; t < kk * kk; t += blockDim.x) gl[t] = __ldcg(G_out + t);
  __syncthreads();
  chol_inverse_block(gl, kk, ri);
  for (int t = threadIdx.x; t < kk * kk; t += blockDim.x) Rinv_out[t] = ri[t];
}

// embedding = (V R^-1)[:, 1:] and max |embedding| for kk > kMaxCols (one warp per row)
__global__ void __launch_bounds__(kBlock) finish_orth_wide_kernel(const float* __restrict__ V,
                                                                  const double* __restrict__ Rinv, int64_t n, int kk,
                                                                  int vp, float* __restrict__ emb,
                                                                  unsigned* __restrict__ absmax) {
  __shared__ double ri[kWideCols * kWideCols];
  for (int t = threadIdx.x; t < kk * kk; t += blockDim.x) ri[t] = Rinv[t];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t r = (int64_t)blockIdx.x * (kBlock / 32) + warp;
  float m = 0.f;
  const double v0 = (r < n && lane < kk) ? (double)V[r * vp + lane] : 0.0;
  const double v1 = (r < n && lane + 32 < kk) ? (double)V[r * vp + lane + 32] : 0.0;
  double q0, q1;
  apply_rinv_wide(v0, v1, ri, kk, lane, q0, q1);
  if (r < n) {
    if (lane >= 1 && lane < kk) {
      const float f = (float)q0;
      emb[r * (kk - 1) + (lane - 1)] = f;
      m = fabsf(f);
    }
    if (lane + 32 < kk) {
      const float f = (float)q1;
      emb[r * (kk - 1) + (lane + 31)] = f;
      m = fmaxf(m, fabsf(f));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) atomicMax(absmax, __float_as_uint(m));
}

// ---- all power iterations in one cooperative launch ---------------------------
// The per-iteration launches above spend most of their time starting and ending
// (100 dependent launches of a few microseconds of work).  Here the grid stays
// resident: each iteration is the SpMV + Gram step of spmv_gram_kernel over a
// grid-stride range of rows, then one grid barrier, after which EVERY block
// factors the completed Gram matrix itself (a few FP64 operations) instead of
// waiting for a last block.  V rows written by other blocks are read through L2
// (ld.global.cg).  The barrier gives up after limit_ns (umapb_set_wait_limit_ns,
// 2 s by default), raises a shared abort flag and the status word, and every
// block then returns.

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ bool grid_barrier(unsigned* bar, unsigned target, int* abort_g, unsigned long long limit_ns) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();
    atomicAdd(bar, 1u);
    const unsigned long long t0 = gtimer();
    for (unsigned i = 1;; ++i) {
      unsigned v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
      if (v >= target) break;
      if ((i & 255) == 0 && *(volatile int*)abort_g) {
        ok = 0;
        break;
      }
      if (gtimer() - t0 > limit_ns) {
        atomicExch(abort_g, 1);
        ok = 0;
        break;
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

template <int KK>  // columns of V: n_components + 1
__global__ void __launch_bounds__(kBlock) power_kernel(float* __restrict__ V0, float* __restrict__ V1,
                                                       const int64_t* __restrict__ row_ptr,
                                                       const int32_t* __restrict__ cols, const float* __restrict__ wn,
                                                       int64_t n, int n_iter, double* __restrict__ G,
                                                       double* __restrict__ Rinv, unsigned* __restrict__ bar,
                                                       int* __restrict__ abort_g, int32_t* __restrict__ status,
                                                       unsigned long long limit_ns) {
  constexpr int kk = KK;
  constexpr int vp = KK <= 4 ? 4 : 8;
  __shared__ double ri[kMaxCols * kMaxCols];
  __shared__ double gsum[kBlock / 32][kMaxCols * kMaxCols];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sub = threadIdx.x & (kLanes - 1);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x / kLanes;  // rows per grid pass
  if (threadIdx.x < kk * kk) ri[threadIdx.x] = (threadIdx.x % (kk + 1) == 0) ? 1.0 : 0.0;
  __syncthreads();
  for (int it = 0; it < n_iter; ++it) {
    const float* Vin = (it & 1) ? V1 : V0;
    float* Vout = (it & 1) ? V0 : V1;
    double* Git = G + (size_t)it * kk * kk;
    double part[kk * kk];
#pragma unroll
    for (int t = 0; t < kk * kk; ++t) part[t] = 0.0;
    // the loop bound is the warp's first row, so every lane of a warp makes the
    // same passes and meets the shuffle below; rows past n do no work
    for (int64_t r0 = ((int64_t)blockIdx.x * blockDim.x + warp * 32) / kLanes; r0 < n; r0 += stride) {
      const int64_t r = r0 + lane / kLanes;
      const bool valid = r < n;
      double acc[kk];
#pragma unroll
      for (int j = 0; j < kk; ++j) acc[j] = 0.0;
      const int64_t e1 = valid ? row_ptr[r + 1] : 0;
      // one edge's contribution: acc_j += w q_j with q_j = sum_i v_i Rinv[i][j]
      auto add_edge = [&](double w, const float4& a, float a4) {
        double v[kMaxCols];
        v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w;
        if (kk > 4) v[4] = a4;
#pragma unroll
        for (int j = 0; j < kk; ++j) {
          double q = 0.0;
#pragma unroll
          for (int i = 0; i <= j; ++i) q += v[i] * ri[i * kk + j];
          acc[j] += w * q;
        }
      };
      int64_t e = valid ? row_ptr[r] + sub : 0;
      // four edges per step: their column ids, weights and V rows are loaded
      // together (two round trips per four edges); the sums keep edge order
      for (; e + 3 * kLanes < e1; e += 4 * kLanes) {
        int64_t c[4];
        double w[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          c[u] = cols[e + u * kLanes];
          w[u] = (double)wn[e + u * kLanes];
        }
        float4 a[4];
        float a4[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          a[u] = __ldcg(reinterpret_cast<const float4*>(Vin + c[u] * vp));  // rows padded to 4 or 8
          a4[u] = kk > 4 ? __ldcg(Vin + c[u] * vp + 4) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) add_edge(w[u], a[u], a4[u]);
      }
      for (; e < e1; e += kLanes) {
        const int64_t c = cols[e];
        add_edge((double)wn[e], __ldcg(reinterpret_cast<const float4*>(Vin + c * vp)),
                 kk > 4 ? __ldcg(Vin + c * vp + 4) : 0.f);
      }
#pragma unroll
      for (int j = 0; j < kk; ++j) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], 1);  // kLanes == 2
      if (valid && sub == 0) {
#pragma unroll
        for (int j = 0; j < vp; ++j) Vout[r * vp + j] = j < kk ? (float)acc[j] : 0.f;
#pragma unroll
        for (int i = 0; i < kk; ++i)
#pragma unroll
          for (int j = i; j < kk; ++j) part[i * kk + j] += acc[i] * acc[j];
      }
    }
    // block reduction of the Gram partials, then one atomic per entry and block
#pragma unroll
    for (int i = 0; i < kk; ++i) {
#pragma unroll
      for (int j = i; j < kk; ++j) {
        double g = part[i * kk + j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
        if (lane == 0) gsum[warp][i * kk + j] = g;
      }
    }
    __syncthreads();
    if (threadIdx.x < kk * kk) {
      const int i = threadIdx.x / kk, j = threadIdx.x % kk;
      if (i <= j) {
        double g = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) g += gsum[w][i * kk + j];
        atomicAdd(&Git[i * kk + j], g);
        if (i != j) atomicAdd(&Git[j * kk + i], g);
      }
    }
    if (!grid_barrier(bar, (unsigned)(it + 1) * gridDim.x, abort_g, limit_ns)) {
      if (threadIdx.x == 0) atomicExch(status, (int32_t)kDevTimeoutEpilogue);
      return;
    }
    if (threadIdx.x == 0) {
      double Gl[kMaxCols * kMaxCols];
      for (int t = 0; t < kk * kk; ++t) Gl[t] = __ldcg(Git + t);
      double rl[kMaxCols * kMaxCols];
      chol_inverse(Gl, kk, rl);
      for (int t = 0; t < kk * kk; ++t) ri[t] = rl[t];
      if (blockIdx.x == 0)
        for (int t = 0; t < kk * kk; ++t) Rinv[(size_t)it * kk * kk + t] = rl[t];
    }
    __syncthreads();
  }
}

__device__ __forceinline__ unsigned f2ord(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// embedding = (V R^-1)[:, 1:], max |embedding|
__global__ void finish_orth_kernel(const float* __restrict__ V, const double* __restrict__ Rinv, int64_t n, int kk,
                                   int vp, float* __restrict__ emb, unsigned* __restrict__ absmax) {
  __shared__ double ri[kMaxCols * kMaxCols];
  if (threadIdx.x < kk * kk) ri[threadIdx.x] = Rinv[threadIdx.x];
  __syncthreads();
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float m = 0.f;
  if (r < n) {
    for (int j = 1; j < kk; ++j) {
      double q = 0.0;
      for (int i = 0; i <= j; ++i) q += (double)V[r * vp + i] * ri[i * kk + j];
      const float f = (float)q;
      emb[r * (kk - 1) + (j - 1)] = f;
      m = fmaxf(m, fabsf(f));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(absmax, __float_as_uint(m));
}

// e = f32(emb * (10 / max|emb|)) + noise (umap.py:344-346); per-column min/max
__global__ void scale_noise_kernel(float* __restrict__ emb, const float* __restrict__ noise, int64_t n, int dim,
                                   const unsigned* __restrict__ absmax, unsigned* __restrict__ colmin,
                                   unsigned* __restrict__ colmax) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const float expansion = __fdiv_rn(10.0f, __uint_as_float(*absmax));
  if (t < n * dim) {
    const float v = __fadd_rn(__fmul_rn(emb[t], expansion), noise[t]);
    emb[t] = v;
    const int c = (int)(t % dim);
    atomicMin(&colmin[c], f2ord(v));
    atomicMax(&colmax[c], f2ord(v));
  }
}

// Y = 10 (e - min) / (max - min + 1e-10) per column (umap.py:347)
__global__ void minmax_kernel(const float* __restrict__ emb, int64_t n, int dim, const unsigned* __restrict__ colmin,
                              const unsigned* __restrict__ colmax, float* __restrict__ Y) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * dim) return;
  const int c = (int)(t % dim);
  const float mn = ord2f(colmin[c]), mx = ord2f(colmax[c]);
  const float num = __fmul_rn(10.0f, __fsub_rn(emb[t], mn));
  const float den = __fadd_rn(__fsub_rn(mx, mn), 1e-10f);
  Y[t] = __fdiv_rn(num, den);
}

struct Layout {
  int32_t* status;
  int64_t* row_ptr;
  float* dis;
  float* wn;
  float* V[2];  // n rows of vp floats (kk values, zero padded to 4 or 8)
  double* G;       // n_iter blocks of kk*kk
  double* Rinv;    // n_iter blocks of kk*kk: the inverse Cholesky factor after each iteration
  unsigned* done;  // per-iteration block counters; done[n_iter] the grid barrier
  int* abort_g;    // cooperative path: barrier abort flag
  float* emb;
  unsigned* red;  // absmax, colmin[kWideCols], colmax[kWideCols]
  size_t bytes;
};

static int vpitch(int kk) { return kk <= 4 ? 4 : (kk + 3) / 4 * 4; }

static Layout carve(void* ws, int64_t n, int dim, int64_t e_cap, int n_iter) {
  const int kk = dim + 1;
  Carver c(ws);
  Layout l;
  l.status = c.take<int32_t>(64);
  l.row_ptr = c.take<int64_t>((size_t)n + 1);
  l.dis = c.take<float>((size_t)n);
  l.wn = c.take<float>((size_t)(e_cap > 0 ? e_cap : 1));
  l.V[0] = c.take<float>((size_t)n * vpitch(kk));
  l.V[1] = c.take<float>((size_t)n * vpitch(kk));
  l.G = c.take<double>((size_t)(n_iter > 0 ? n_iter : 1) * kk * kk);
  l.Rinv = c.take<double>((size_t)(n_iter > 0 ? n_iter : 1) * kk * kk);
  l.done = c.take<unsigned>((size_t)(n_iter > 0 ? n_iter : 1) + 1);
  l.abort_g = c.take<int>(1);
  l.emb = c.take<float>((size_t)n * dim);
  l.red = c.take<unsigned>(1 + 2 * kWideCols);
  l.bytes = c.bytes();
  return l;
}

// V0 (n x kk) into rows of vp floats, zero padded
__global__ void pad_rows_kernel(const float* __restrict__ a, int64_t n, int kk, int vp, float* __restrict__ b) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * vp) return;
  const int64_t r = t / vp;
  const int j = (int)(t - r * vp);
  b[t] = j < kk ? a[r * kk + j] : 0.f;
}

// Standard normal draws: element i of the stream (seed) comes from Philox block i/4
// and the Box-Muller transform of its two 32-bit pairs.
__device__ __forceinline__ void normal4(int64_t blk, uint32_t k0, uint32_t k1, float (&z)[4]) {
  const U4 r = philox4x32_10(U4{(uint32_t)blk, (uint32_t)(blk >> 32), 0x5eedu, 0u}, k0, k1);
  float s0, c0, s1, c1;
  const float r0 = sqrtf(-2.0f * logf(to_unit(r.x)));
  const float r1 = sqrtf(-2.0f * logf(to_unit(r.z)));
  sincospif(2.0f * to_unit(r.y), &s0, &c0);
  sincospif(2.0f * to_unit(r.w), &s1, &c1);
  z[0] = r0 * c0, z[1] = r0 * s0, z[2] = r1 * c1, z[3] = r1 * s1;
}

__global__ void normal_fill_kernel(float* __restrict__ out, int64_t count, uint32_t k0, uint32_t k1) {
  const int64_t blk = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (blk * 4 >= count) return;
  float z[4];
  normal4(blk, k0, k1, z);
  for (int u = 0; u < 4; ++u)
    if (blk * 4 + u < count) out[blk * 4 + u] = z[u];
}

__global__ void init_red_kernel(unsigned* red, int dim) {
  if (threadIdx.x == 0) red[0] = 0u;
  if (threadIdx.x < (unsigned)dim) {
    red[1 + threadIdx.x] = 0xFFFFFFFFu;          // min
    red[1 + kWideCols + threadIdx.x] = 0u;       // max
  }
}

// The reference falls back to a random start when its spectral init fails
// (umap.py:354-357).  When the power iteration's grid barrier gave up (status word
// non-zero), Y is replaced on the device by N(0, 1) * 0.01 drawn from the Philox
// stream of umapb_normal_fill(seed), so no host round trip sits between the
// spectral init and the layout.
__global__ void fallback_kernel(const int32_t* __restrict__ status, float* __restrict__ Y, int64_t count,
                                uint32_t k0, uint32_t k1) {
  if (*status == 0) return;
  const int64_t blk = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (blk * 4 >= count) return;
  float z[4];
  normal4(blk, k0, k1, z);
  for (int u = 0; u < 4; ++u)
    if (blk * 4 + u < count) Y[blk * 4 + u] = __fmul_rn(z[u], 0.01f);
}

}  // namespace spectral
}  // namespace umapb

using namespace umapb;

extern "C" int umapb_spectral_workspace(int64_t n, int32_t dim, int64_t e_cap, int32_t n_iter, size_t* bytes) {
  clear_error();
  UMAPB_REQUIRE(bytes, "bytes is null");
  UMAPB_REQUIRE(n >= 1 && dim >= 1 && dim <= 32, "spectral: need n >= 1 and 1 <= dim <= 32");
  UMAPB_REQUIRE(n_iter >= 1 && n_iter <= 128, "spectral: need 1 <= n_iter <= 128");
  UMAPB_REQUIRE(e_cap >= 0, "spectral: e_cap must be >= 0");
  *bytes = spectral::carve(nullptr, n, dim, e_cap, n_iter).bytes;
  return UMAPB_OK;
}

extern "C" int umapb_spectral(const int32_t* rows, const int32_t* cols, const float* vals, const int64_t* n_edges,
                              int64_t e_cap, int64_t n, int32_t dim, const float* V0, int32_t n_iter,
                              const float* noise, float* Y, void* workspace, size_t workspace_bytes,
                              umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(rows && cols && vals && n_edges && V0 && noise && Y, "spectral: null array argument");
  UMAPB_REQUIRE(n >= 1 && dim >= 1 && dim <= 32, "spectral: need n >= 1 and 1 <= dim <= 32");
  UMAPB_REQUIRE(n_iter >= 1 && n_iter <= 128, "spectral: need 1 <= n_iter <= 128");
  UMAPB_REQUIRE(e_cap >= 0, "spectral: e_cap must be >= 0");
  spectral::Layout l = spectral::carve(nullptr, n, dim, e_cap, n_iter);
  if (!workspace || workspace_bytes < l.bytes)
    return set_error(UMAPB_ERR_WORKSPACE, "spectral: workspace of %zu bytes, need %zu", workspace_bytes, l.bytes);
  l = spectral::carve(workspace, n, dim, e_cap, n_iter);
  const int kk = dim + 1;
  const unsigned rb = (unsigned)ceil_div(n, spectral::kBlock);
  UMAPB_CUDA_TRY(cudaMemsetAsync(l.status, 0, 4, stream), "spectral: status reset");
  UMAPB_CUDA_TRY(cudaMemsetAsync(l.G, 0, sizeof(double) * n_iter * kk * kk, stream), "spectral: gram reset");
  UMAPB_CUDA_TRY(cudaMemsetAsync(l.done, 0, sizeof(unsigned) * (n_iter + 1), stream), "spectral: counter reset");
  UMAPB_CUDA_TRY(cudaMemsetAsync(l.abort_g, 0, sizeof(int), stream), "spectral: abort reset");
  spectral::row_ptr_kernel<<<(unsigned)ceil_div(n + 1, spectral::kBlock), spectral::kBlock, 0, stream>>>(
      rows, n_edges, n, l.row_ptr);
  spectral::degree_kernel<<<rb, spectral::kBlock, 0, stream>>>(vals, l.row_ptr, n, l.dis);
  if (e_cap > 0)
    spectral::norm_weight_kernel<<<(unsigned)ceil_div(e_cap, spectral::kBlock), spectral::kBlock, 0, stream>>>(
        rows, cols, vals, n_edges, l.dis, l.wn);
  const int vp = spectral::vpitch(kk);
  spectral::pad_rows_kernel<<<(unsigned)ceil_div(n * vp, spectral::kBlock), spectral::kBlock, 0, stream>>>(
      V0, n, kk, vp, l.V[0]);
  UMAPB_LAUNCH_CHECK("spectral: setup kernels");
  const unsigned pb = (unsigned)ceil_div(n * spectral::kLanes, spectral::kBlock);
  // one cooperative launch for all iterations (every block resident), sized to
  // the rows; the per-iteration launches remain for devices that refuse it and
  // behind UMAPB_SPECTRAL_COOP=0
  int per_sm = 0;
  int coop = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  {
    const char* e = getenv("UMAPB_SPECTRAL_COOP");
    if (e && e[0] == '0' && e[1] == 0) coop = 0;
  }
  const void* pk = kk == 2   ? (const void*)spectral::power_kernel<2>
                   : kk == 3 ? (const void*)spectral::power_kernel<3>
                   : kk == 4 ? (const void*)spectral::power_kernel<4>
                             : (const void*)spectral::power_kernel<5>;
  if (coop && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pk, spectral::kBlock, 0) != cudaSuccess)
    per_sm = 0;
  cudaGetLastError();
  int64_t grid = (int64_t)num_sms() * (per_sm < 4 ? per_sm : 4);
  if (grid > (int64_t)pb) grid = pb;
  bool launched = false;
  const bool wide = kk > spectral::kMaxCols;
  if (wide) coop = 0;
  if (coop && grid > 0) {
    float* v0 = l.V[0];
    float* v1 = l.V[1];
    const int64_t* rp = l.row_ptr;
    const float* w = l.wn;
    int64_t nn = n;
    int ni = n_iter;
    double* G = l.G;
    double* R = l.Rinv;
    unsigned* bar = l.done + n_iter;
    int* ab = l.abort_g;
    int32_t* st = l.status;
    unsigned long long lim = wait_limit_ns();
    void* args[] = {&v0, &v1, &rp, &cols, &w, &nn, &ni, &G, &R, &bar, &ab, &st, &lim};
    launched = cudaLaunchCooperativeKernel(pk, dim3((unsigned)grid), dim3(spectral::kBlock), args, 0, stream) ==
               cudaSuccess;
    if (!launched) cudaGetLastError();
  }
  if (!launched && wide) {
    const unsigned wb = (unsigned)ceil_div(n, spectral::kWideRows);
    for (int it = 0; it < n_iter; ++it) {
      const double* rprev = it == 0 ? nullptr : l.Rinv + (size_t)(it - 1) * kk * kk;
      spectral::spmv_gram_wide_kernel<<<wb, spectral::kBlock, 0, stream>>>(
          l.V[it & 1], rprev, l.row_ptr, cols, l.wn, n, kk, vp, l.V[(it + 1) & 1], l.G + (size_t)it * kk * kk,
          l.done + it, l.Rinv + (size_t)it * kk * kk);
    }
  } else if (!launched) {
    for (int it = 0; it < n_iter; ++it) {
      const double* rprev = it == 0 ? nullptr : l.Rinv + (size_t)(it - 1) * kk * kk;
      spectral::spmv_gram_kernel<<<pb, spectral::kBlock, 0, stream>>>(
          l.V[it & 1], rprev, l.row_ptr, cols, l.wn, n, kk, vp, l.V[(it + 1) & 1], l.G + (size_t)it * kk * kk,
          l.done + it, l.Rinv + (size_t)it * kk * kk);
    }
  }
  UMAPB_LAUNCH_CHECK("spectral: power iteration");
  spectral::init_red_kernel<<<1, 32, 0, stream>>>(l.red, dim);
  if (wide)
    spectral::finish_orth_wide_kernel<<<(unsigned)ceil_div(n, spectral::kBlock / 32), spectral::kBlock, 0, stream>>>(
        l.V[n_iter & 1], l.Rinv + (size_t)(n_iter - 1) * kk * kk, n, kk, vp, l.emb, l.red);
  else
    spectral::finish_orth_kernel<<<rb, spectral::kBlock, 0, stream>>>(l.V[n_iter & 1],
                                                                       l.Rinv + (size_t)(n_iter - 1) * kk * kk, n,
                                                                       kk, vp, l.emb, l.red);
  const unsigned eb = (unsigned)ceil_div(n * dim, spectral::kBlock);
  unsigned* colmin = l.red + 1;
  unsigned* colmax = l.red + 1 + spectral::kWideCols;
  spectral::scale_noise_kernel<<<eb, spectral::kBlock, 0, stream>>>(l.emb, noise, n, dim, l.red, colmin, colmax);
  spectral::minmax_kernel<<<eb, spectral::kBlock, 0, stream>>>(l.emb, n, dim, colmin, colmax, Y);
  UMAPB_LAUNCH_CHECK("spectral: rescale kernels");
  count_launches((e_cap > 0 ? 3 : 2) + 1 + (launched ? 1 : n_iter) + 4);
  return UMAPB_OK;
}

extern "C" int umapb_spectral_fallback(const void* workspace, float* Y, int64_t n, int32_t dim, uint64_t seed,
                                       umapb_stream_t stream_) {
  clear_error();
  UMAPB_REQUIRE(workspace && Y, "spectral_fallback: null argument");
  UMAPB_REQUIRE(n >= 1 && dim >= 1 && dim <= 32, "spectral_fallback: need n >= 1 and 1 <= dim <= 32");
  const int64_t count = n * dim;
  const int64_t blocks4 = ceil_div(count, 4);
  spectral::fallback_kernel<<<(unsigned)ceil_div(blocks4, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream_)>>>(
      static_cast<const int32_t*>(workspace), Y, count, (uint32_t)seed, (uint32_t)(seed >> 32));
  UMAPB_LAUNCH_CHECK("spectral_fallback kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_normal_fill(float* out, int64_t count, uint64_t seed, umapb_stream_t stream_) {
  clear_error();
  UMAPB_REQUIRE(out || count == 0, "normal_fill: null output");
  UMAPB_REQUIRE(count >= 0, "normal_fill: count must be >= 0");
  if (count == 0) return UMAPB_OK;
  const int64_t blocks4 = ceil_div(count, 4);
  spectral::normal_fill_kernel<<<(unsigned)ceil_div(blocks4, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream_)>>>(
      out, count, (uint32_t)seed, (uint32_t)(seed >> 32));
  UMAPB_LAUNCH_CHECK("normal_fill kernel");
  count_launches(1);
  return UMAPB_OK;
}
