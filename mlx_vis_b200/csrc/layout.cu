// Layout optimisation — replaces UMAP._optimize and UMAP._sgd_step,
// mlx_vis/_umap/umap.py:359-449.
//
// Schedule (umap.py:398-414): eps_e = n_epochs / (n_epochs * (w_e / max w)) in
// float32, next_e starts at eps_e; edge e is active in epoch t when
// next_e <= t, after which next_e += eps_e (float32).  The reference builds all
// active sets on the host up front; here every epoch kernel re-evaluates the
// same float32 recurrence per edge, so the sets are identical and no host work
// or per-epoch index list is needed.
//
// Epoch (umap.py:359-387): every gather reads the epoch-start Y; the moves of
// all pairs are accumulated into dY with float atomics and applied by a second
// kernel, which reproduces the reference's synchronous scatter-add semantics.
// Per active edge (i, j): attractive move clip(-2ab d^{2(b-1)}/(1+a d^{2b}) diff,
// +-4) * alpha added to i and subtracted from j; neg_rate negatives (i, t) each
// add clip(2b/((0.001+d^2)(1+a d^{2b})) diff, +-4) * alpha to i only.  The moves
// of one edge on its head are summed in registers before one atomic.
//
// Negatives: the reference pairs sample s of an epoch with head ef[s % A] and a
// uniform tail from mx.random.randint (umap.py:433-436).  The fast path draws
// the tail of (epoch, edge e, sample m) from Philox4x32-10 (Salmon et al., SC'11)
// keyed by the seed, mapped to [0, n) by a 32x32->64 multiply-high (bias below
// n / 2^32).  The injected path takes the reference's own tails: it ranks the
// active edges in edge order (block counts + scan) and uses tail neg_to[r + m A]
// for the r-th active edge.
#include <math.h>
#include <stdlib.h>

#include <mutex>

#include "common.cuh"
#include "philox.cuh"
#include "scan.cuh"

namespace umapb {
namespace layout {

constexpr int kBlock = 256;
constexpr int kEdgesPerBlock = 1024;
#ifndef UMAPB_LAYOUT_BLOCKS_PER_SM
#define UMAPB_LAYOUT_BLOCKS_PER_SM 4
#endif
// resident blocks per SM the epoch kernel is compiled for (register cap) and launched with
constexpr int kEpochBlocksPerSM = UMAPB_LAYOUT_BLOCKS_PER_SM;
#ifndef UMAPB_LAYOUT_BLOCKS_PER_SM5
#define UMAPB_LAYOUT_BLOCKS_PER_SM5 4
#endif
// the same for the kernel specialised to 5 negatives per edge (the default rate)
constexpr int kEpochBlocksPerSM5 = UMAPB_LAYOUT_BLOCKS_PER_SM5;
constexpr int kPre = 8;  // epoch kernel: chunks of 32 edges whose schedule words load together

// ---- reference pair math (float32, evaluation order of umap.py:361-383) ----
struct Params {
  float a, b, m2ab, two_b, alpha;
};

// d^(2b) is evaluated once per pair as exp2(b log2 d2) (CUDA's log2f / exp2f, a few
// ulp); d^(2(b-1)) = d^(2b) / d2.  The reference evaluates mx.power twice in float32;
// the difference is a few float32 ulp of the coefficient.
__device__ __forceinline__ float pow_b(float d2, float b) { return exp2f(__fmul_rn(b, log2f(d2))); }

template <int DIM>
__device__ __forceinline__ void attract(const float (&yi)[DIM], const float (&yj)[DIM], const Params& p,
                                        float (&out)[DIM]) {
  float diff[DIM];
  float d2 = 0.f;
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    diff[c] = __fsub_rn(yi[c], yj[c]);
    d2 = __fadd_rn(d2, __fmul_rn(diff[c], diff[c]));
  }
  d2 = fmaxf(d2, 1e-6f);
  const float pw = pow_b(d2, p.b);
  // -2ab d^(2(b-1)) / (1 + a d^(2b)) = (-2ab) d^(2b) / (d2 (1 + a d^(2b)))
  const float coeff = __fdiv_rn(__fmul_rn(p.m2ab, pw), __fmul_rn(d2, __fadd_rn(1.0f, __fmul_rn(p.a, pw))));
#pragma unroll
  for (int c = 0; c < DIM; ++c) out[c] = __fmul_rn(fminf(fmaxf(__fmul_rn(coeff, diff[c]), -4.0f), 4.0f), p.alpha);
}

template <int DIM>
__device__ __forceinline__ void repel_add(const float (&yi)[DIM], const float (&yt)[DIM], const Params& p,
                                          float (&acc)[DIM]) {
  float diff[DIM];
  float d2 = 0.f;
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    diff[c] = __fsub_rn(yi[c], yt[c]);
    d2 = __fadd_rn(d2, __fmul_rn(diff[c], diff[c]));
  }
  d2 = fmaxf(d2, 1e-6f);
  const float pw = pow_b(d2, p.b);
  const float den = __fmul_rn(__fadd_rn(0.001f, d2), __fadd_rn(1.0f, __fmul_rn(p.a, pw)));
  const float coeff = __fdiv_rn(p.two_b, den);
#pragma unroll
  for (int c = 0; c < DIM; ++c)
    acc[c] = __fadd_rn(acc[c], __fmul_rn(fminf(fmaxf(__fmul_rn(coeff, diff[c]), -4.0f), 4.0f), p.alpha));
}

template <int DIM>
__device__ __forceinline__ void load_row(const float* __restrict__ Y, int i, float (&v)[DIM]) {
  if constexpr (DIM == 2) {
    const float2 t = __ldg(reinterpret_cast<const float2*>(Y) + i);
    v[0] = t.x;
    v[1] = t.y;
  } else if constexpr (DIM == 4) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(Y) + i);
    v[0] = t.x;
    v[1] = t.y;
    v[2] = t.z;
    v[3] = t.w;
  } else {
#pragma unroll
    for (int c = 0; c < DIM; ++c) v[c] = __ldg(Y + (int64_t)i * DIM + c);
  }
}

template <int DIM>
__device__ __forceinline__ void atomic_add_row(float* __restrict__ dY, int i, const float (&v)[DIM]) {
  if constexpr (DIM == 2) {
    atomicAdd(reinterpret_cast<float2*>(dY) + i, make_float2(v[0], v[1]));
  } else if constexpr (DIM == 4) {
    atomicAdd(reinterpret_cast<float4*>(dY) + i, make_float4(v[0], v[1], v[2], v[3]));
  } else {
#pragma unroll
    for (int c = 0; c < DIM; ++c) atomicAdd(dY + (int64_t)i * DIM + c, v[c]);
  }
}

// ---- schedule ----------------------------------------------------------------
__global__ void max_kernel(const float* __restrict__ vals, const int64_t* __restrict__ n_edges, float* __restrict__ wmax) {
  const int64_t E = *n_edges;
  float m = 0.f;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x)
    m = fmaxf(m, vals[e]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int*>(wmax), __float_as_int(m));
}

__global__ void eps_kernel(const float* __restrict__ vals, const int64_t* __restrict__ n_edges,
                           const float* __restrict__ wmax, int n_epochs, float* __restrict__ eps,
                           float* __restrict__ next) {
  const int64_t E = *n_edges;
  const float wm = *wmax;
  const float ne = (float)n_epochs;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
    const float ns = __fmul_rn(ne, __fdiv_rn(vals[e], wm));
    const float v = ns > 0.f ? __fdiv_rn(ne, ns) : -1.0f;
    eps[e] = v;
    next[e] = v;
  }
}

// ---- fast path epoch ---------------------------------------------------------
// Only the edges due in an epoch do work, about a third of them on average, so a
// thread-per-edge loop leaves most lanes idle.  Each warp scans a contiguous
// segment of edges, advances the schedule of the due ones and queues them in
// shared memory; the warp works through the queue 32 edges at a time with every
// lane busy (at most one partial batch per warp, at the end of its segment).
// NEG > 0: compiled for exactly NEG (<= 8) negatives per edge (neg_rate == NEG), so
// the registers of the unused sample slots are not held.
template <int DIM, int NEG>
__device__ __forceinline__ void edge_update(const float* __restrict__ Y, float* __restrict__ dY, int n, int i,
                                            int j, int64_t e, int epoch, const Params& p, int neg_rate, uint32_t k0,
                                            uint32_t k1) {
  static_assert(NEG >= 0 && NEG <= 8, "NEG is 0 (any rate) or a rate <= 8");
  float yi[DIM], yj[DIM], acc[DIM], pos[DIM], neg_pos[DIM];
  constexpr int kSlots = NEG > 0 ? NEG : 8;
  const int nr = NEG > 0 ? NEG : neg_rate;
  if (NEG > 0 || neg_rate <= 8) {
    // up to 8 negatives: draw their tails and issue every gather of Y before the
    // arithmetic, so the seven or so random reads of an edge are in flight together
    const U4 r0 = philox4x32_10(U4{(uint32_t)e, (uint32_t)(e >> 32), (uint32_t)epoch, 0u}, k0, k1);
    U4 r1 = r0;
    if (nr > 4) r1 = philox4x32_10(U4{(uint32_t)e, (uint32_t)(e >> 32), (uint32_t)epoch, 1u}, k0, k1);
    const uint32_t rr[8] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
    float yt[kSlots][DIM];
    load_row<DIM>(Y, i, yi);
    load_row<DIM>(Y, j, yj);
#pragma unroll
    for (int u = 0; u < kSlots; ++u)
      if (u < nr) load_row<DIM>(Y, to_range(rr[u], (uint32_t)n), yt[u]);
    attract<DIM>(yi, yj, p, pos);
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      acc[c] = pos[c];
      neg_pos[c] = -pos[c];
    }
#pragma unroll
    for (int u = 0; u < kSlots; ++u)
      if (u < nr) repel_add<DIM>(yi, yt[u], p, acc);
    atomic_add_row<DIM>(dY, j, neg_pos);
    atomic_add_row<DIM>(dY, i, acc);
    return;
  }
  load_row<DIM>(Y, i, yi);
  load_row<DIM>(Y, j, yj);
  attract<DIM>(yi, yj, p, pos);
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    acc[c] = pos[c];
    neg_pos[c] = -pos[c];
  }
  atomic_add_row<DIM>(dY, j, neg_pos);
  auto repel = [&](uint32_t r) {
    float yt[DIM];
    load_row<DIM>(Y, to_range(r, (uint32_t)n), yt);
    repel_add<DIM>(yi, yt, p, acc);
  };
#pragma unroll 1
  for (int m0 = 0; m0 < neg_rate; m0 += 4) {
    const U4 r = philox4x32_10(U4{(uint32_t)e, (uint32_t)(e >> 32), (uint32_t)epoch, (uint32_t)(m0 >> 2)}, k0, k1);
    repel(r.x);
    if (m0 + 1 < neg_rate) repel(r.y);
    if (m0 + 2 < neg_rate) repel(r.z);
    if (m0 + 3 < neg_rate) repel(r.w);
  }
  atomic_add_row<DIM>(dY, i, acc);
}

template <int DIM, int NEG>
__global__ void __launch_bounds__(kBlock, NEG == 5 ? kEpochBlocksPerSM5 : kEpochBlocksPerSM) sgd_epoch_kernel(const float* __restrict__ Y, float* __restrict__ dY, int n,
                                                           const int32_t* __restrict__ rows,
                                                           const int32_t* __restrict__ cols,
                                                           const float* __restrict__ eps, float* __restrict__ next,
                                                           const int64_t* __restrict__ n_edges, int epoch, Params p,
                                                           int neg_rate, uint32_t k0, uint32_t k1) {
  // A pass: every warp loads the schedule words of kPre chunks of 32 edges of its
  // segment at once (one round trip instead of kPre), advances the due edges and
  // appends them to the block's queue; then the block's 8 warps take the queue 32
  // edges at a time, so only the block's last batch of the pass runs partly empty.
  __shared__ int32_t bq[(kBlock / 32) * kPre * 32];
  __shared__ int s_cnt;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t E = *n_edges;
  const float ep = (float)epoch;
  const int64_t n_warps = (int64_t)gridDim.x * (kBlock / 32);
  const int64_t seg = (((E + 31) / 32 + n_warps - 1) / n_warps) * 32;
  const int64_t b0 = (int64_t)blockIdx.x * (kBlock / 32) * seg;
  const int64_t e0 = b0 + (int64_t)warp * seg;
  const int64_t e1 = e0 + seg < E ? e0 + seg : E;
  const unsigned below = (1u << lane) - 1u;
  const int passes = (int)((seg + 32 * kPre - 1) / (32 * kPre));  // the same for every warp of the grid
  for (int ps = 0; ps < passes; ++ps) {
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    const int64_t sb = e0 + (int64_t)ps * 32 * kPre;
    float nx[kPre], ex[kPre];
#pragma unroll
    for (int u = 0; u < kPre; ++u) {
      const int64_t e = sb + 32 * u + lane;
      nx[u] = e < e1 ? next[e] : INFINITY;
      ex[u] = e < e1 ? eps[e] : 0.f;
    }
#pragma unroll
    for (int u = 0; u < kPre; ++u) {
      const int64_t e = sb + 32 * u + lane;
      const bool due = nx[u] <= ep;
      if (due) next[e] = __fadd_rn(nx[u], ex[u]);
      const unsigned b = __ballot_sync(0xffffffffu, due);
      int slot = 0;
      if (lane == 0 && b) slot = atomicAdd(&s_cnt, __popc(b));
      slot = __shfl_sync(0xffffffffu, slot, 0);
      if (due) bq[slot + __popc(b & below)] = (int32_t)(e - b0);
    }
    __syncthreads();
    // the warp's batches: the head and tail ids of the next batch load while this
    // batch's rows of Y are gathered, one round trip per batch instead of two
    const int total = s_cnt;
    int base = warp * 32;
    int64_t e = 0;
    int i = 0, j = 0;
    if (base + lane < total) {
      e = b0 + bq[base + lane];
      i = rows[e];
      j = cols[e];
    }
    for (; base < total; base += kBlock) {
      const int nb = base + kBlock;
      int64_t e2 = 0;
      int i2 = 0, j2 = 0;
      if (nb + lane < total) {
        e2 = b0 + bq[nb + lane];
        i2 = rows[e2];
        j2 = cols[e2];
      }
      if (base + lane < total) edge_update<DIM, NEG>(Y, dY, n, i, j, e, epoch, p, neg_rate, k0, k1);
      e = e2;
      i = i2;
      j = j2;
    }
    __syncthreads();
  }
}

__global__ void apply_kernel(float* __restrict__ Y, float* __restrict__ dY, int64_t m) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < m; t += (int64_t)gridDim.x * blockDim.x) {
    Y[t] = __fadd_rn(Y[t], dY[t]);
    dY[t] = 0.f;
  }
}

// ---- injected path (reference-ordered negatives) ------------------------------
__global__ void count_active_kernel(const float* __restrict__ next, const int64_t* __restrict__ n_edges, int epoch,
                                    int32_t* __restrict__ block_counts) {
  __shared__ int warp_counts[kBlock / 32];
  const int64_t E = *n_edges;
  const float ep = (float)epoch;
  const int64_t base = (int64_t)blockIdx.x * kEdgesPerBlock;
  int c = 0;
  for (int u = 0; u < kEdgesPerBlock / kBlock; ++u) {
    const int64_t e = base + u * kBlock + threadIdx.x;
    c += (e < E && next[e] <= ep) ? 1 : 0;
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

template <int DIM>
__global__ void __launch_bounds__(kBlock) sgd_injected_kernel(
    const float* __restrict__ Y, float* __restrict__ dY, const int32_t* __restrict__ rows,
    const int32_t* __restrict__ cols, const float* __restrict__ eps, float* __restrict__ next,
    const int64_t* __restrict__ n_edges, int epoch, Params p, int neg_rate, const int32_t* __restrict__ neg_to,
    const int32_t* __restrict__ block_offsets, const int64_t* __restrict__ n_active) {
  __shared__ int warp_base[kBlock / 32];
  __shared__ int running;
  const int64_t E = *n_edges;
  const int64_t A = *n_active;
  const float ep = (float)epoch;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) running = block_offsets[blockIdx.x];
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kEdgesPerBlock;
  for (int u = 0; u < kEdgesPerBlock / kBlock; ++u) {
    const int64_t e = base + u * kBlock + threadIdx.x;
    const float nx = e < E ? next[e] : 1.0f;
    const bool act = e < E && nx <= ep;
    const unsigned ballot = __ballot_sync(0xffffffffu, act);
    if (lane == 0) warp_base[warp] = __popc(ballot);
    __syncthreads();
    if (threadIdx.x == 0) {
      int s = running;
      for (int w = 0; w < kBlock / 32; ++w) {
        const int c = warp_base[w];
        warp_base[w] = s;
        s += c;
      }
      running = s;
    }
    __syncthreads();
    if (act) {
      const int64_t rank = warp_base[warp] + __popc(ballot & ((1u << lane) - 1u));
      next[e] = __fadd_rn(nx, eps[e]);
      const int i = rows[e], j = cols[e];
      float yi[DIM], yj[DIM], acc[DIM], pos[DIM], neg_pos[DIM];
      load_row<DIM>(Y, i, yi);
      load_row<DIM>(Y, j, yj);
      attract<DIM>(yi, yj, p, pos);
#pragma unroll
      for (int c = 0; c < DIM; ++c) {
        acc[c] = pos[c];
        neg_pos[c] = -pos[c];
      }
      atomic_add_row<DIM>(dY, j, neg_pos);
      for (int m = 0; m < neg_rate; ++m) {
        float yt[DIM];
        load_row<DIM>(Y, neg_to[rank + (int64_t)m * A], yt);
        repel_add<DIM>(yi, yt, p, acc);
      }
      atomic_add_row<DIM>(dY, i, acc);
    }
    __syncthreads();
  }
}

// ---- n_components 5..32: one warp per edge, lane c holds component c ---------
// The same pair formulas as attract / repel_add; |diff|^2 is summed across the warp
// (butterfly), so its float32 rounding order differs from the sequential sum of the
// narrow kernels by a few ulp.
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = __fadd_rn(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ float attract_wide(float yi, float yj, const Params& p) {
  const float diff = __fsub_rn(yi, yj);
  const float d2 = fmaxf(warp_sum(__fmul_rn(diff, diff)), 1e-6f);
  const float pw = pow_b(d2, p.b);
  const float coeff = __fdiv_rn(__fmul_rn(p.m2ab, pw), __fmul_rn(d2, __fadd_rn(1.0f, __fmul_rn(p.a, pw))));
  return __fmul_rn(fminf(fmaxf(__fmul_rn(coeff, diff), -4.0f), 4.0f), p.alpha);
}

__device__ __forceinline__ float repel_wide(float yi, float yt, const Params& p) {
  const float diff = __fsub_rn(yi, yt);
  const float d2 = fmaxf(warp_sum(__fmul_rn(diff, diff)), 1e-6f);
  const float pw = pow_b(d2, p.b);
  const float den = __fmul_rn(__fadd_rn(0.001f, d2), __fadd_rn(1.0f, __fmul_rn(p.a, pw)));
  const float coeff = __fdiv_rn(p.two_b, den);
  return __fmul_rn(fminf(fmaxf(__fmul_rn(coeff, diff), -4.0f), 4.0f), p.alpha);
}

// One active edge by a whole warp.  Tails: Philox words of counter (e, epoch, m/4)
// in the order of the narrow kernels; with neg_to, the injected tails of rank `rank`.
__device__ __forceinline__ void edge_update_wide(const float* __restrict__ Y, float* __restrict__ dY, int n, int dim,
                                                 int lane, int i, int j, int64_t e, int epoch, const Params& p,
                                                 int neg_rate, uint32_t k0, uint32_t k1,
                                                 const int32_t* __restrict__ neg_to, int64_t rank, int64_t A) {
  const bool on = lane < dim;
  const float yi = on ? __ldg(Y + (int64_t)i * dim + lane) : 0.f;
  const float yj = on ? __ldg(Y + (int64_t)j * dim + lane) : 0.f;
  const float pos = attract_wide(yi, yj, p);
  if (on) atomicAdd(dY + (int64_t)j * dim + lane, -pos);
  float acc = pos;
  for (int m0 = 0; m0 < neg_rate; m0 += 4) {
    uint32_t r[4];
    if (!neg_to) {
      const U4 q = philox4x32_10(U4{(uint32_t)e, (uint32_t)(e >> 32), (uint32_t)epoch, (uint32_t)(m0 >> 2)}, k0, k1);
      r[0] = q.x, r[1] = q.y, r[2] = q.z, r[3] = q.w;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (m0 + u >= neg_rate) break;
      const int t = neg_to ? neg_to[rank + (int64_t)(m0 + u) * A] : to_range(r[u], (uint32_t)n);
      const float yt = on ? __ldg(Y + (int64_t)t * dim + lane) : 0.f;
      acc = __fadd_rn(acc, repel_wide(yi, yt, p));
    }
  }
  if (on) atomicAdd(dY + (int64_t)i * dim + lane, acc);
}

__global__ void __launch_bounds__(kBlock) sgd_epoch_wide_kernel(const float* __restrict__ Y, float* __restrict__ dY,
                                                                int n, int dim, const int32_t* __restrict__ rows,
                                                                const int32_t* __restrict__ cols,
                                                                const float* __restrict__ eps,
                                                                float* __restrict__ next,
                                                                const int64_t* __restrict__ n_edges, int epoch,
                                                                Params p, int neg_rate, uint32_t k0, uint32_t k1) {
  const int lane = threadIdx.x & 31;
  const int64_t E = *n_edges;
  const float ep = (float)epoch;
  const int64_t warps = (int64_t)gridDim.x * (kBlock / 32);
  for (int64_t base = ((int64_t)blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5)) * 32; base < E; base += warps * 32) {
    const int64_t e = base + lane;
    bool due = false;
    if (e < E) {
      const float nx = next[e];
      due = nx <= ep;
      if (due) next[e] = __fadd_rn(nx, eps[e]);
    }
    unsigned b = __ballot_sync(0xffffffffu, due);
    while (b) {
      const int t = __ffs(b) - 1;
      b &= b - 1;
      const int64_t ed = base + t;
      edge_update_wide(Y, dY, n, dim, lane, rows[ed], cols[ed], ed, epoch, p, neg_rate, k0, k1, nullptr, 0, 0);
    }
  }
}

// Injected tails for n_components 5..32: active edges of each 256-edge chunk are
// ranked like sgd_injected_kernel (block offsets from the scan), queued in shared
// memory, and each queued edge is processed by one warp.
__global__ void __launch_bounds__(kBlock) sgd_injected_wide_kernel(
    const float* __restrict__ Y, float* __restrict__ dY, int n, int dim, const int32_t* __restrict__ rows,
    const int32_t* __restrict__ cols, const float* __restrict__ eps, float* __restrict__ next,
    const int64_t* __restrict__ n_edges, int epoch, Params p, int neg_rate, const int32_t* __restrict__ neg_to,
    const int32_t* __restrict__ block_offsets, const int64_t* __restrict__ n_active) {
  __shared__ int warp_base[kBlock / 32];
  __shared__ int running;
  __shared__ int64_t q_edge[kBlock];
  __shared__ int64_t q_rank[kBlock];
  __shared__ int chunk_start, chunk_count;
  const int64_t E = *n_edges;
  const int64_t A = *n_active;
  const float ep = (float)epoch;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) running = block_offsets[blockIdx.x];
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kEdgesPerBlock;
  for (int u = 0; u < kEdgesPerBlock / kBlock; ++u) {
    const int64_t e = base + u * kBlock + threadIdx.x;
    const float nx = e < E ? next[e] : 1.0f;
    const bool act = e < E && nx <= ep;
    const unsigned ballot = __ballot_sync(0xffffffffu, act);
    if (lane == 0) warp_base[warp] = __popc(ballot);
    __syncthreads();
    if (threadIdx.x == 0) {
      int s = running;
      chunk_start = s;
      for (int w = 0; w < kBlock / 32; ++w) {
        const int c = warp_base[w];
        warp_base[w] = s;
        s += c;
      }
      chunk_count = s - running;
      running = s;
    }
    __syncthreads();
    if (act) {
      const int64_t rank = warp_base[warp] + __popc(ballot & ((1u << lane) - 1u));
      next[e] = __fadd_rn(nx, eps[e]);
      q_edge[rank - chunk_start] = e;
      q_rank[rank - chunk_start] = rank;
    }
    __syncthreads();
    for (int t = warp; t < chunk_count; t += kBlock / 32) {
      const int64_t ed = q_edge[t];
      edge_update_wide(Y, dY, n, dim, lane, rows[ed], cols[ed], ed, epoch, p, neg_rate, 0, 0, neg_to, q_rank[t], A);
    }
    __syncthreads();
  }
}

struct Layout {
  int32_t* status;
  float* dY;
  float* wmax;
  int32_t* block_counts;
  int64_t* total;
  int64_t* scan_ws;  // scan_exclusive's block totals
  size_t bytes;
};

static Layout carve(void* ws, int64_t n, int dim, int64_t e_cap) {
  Carver c(ws);
  Layout l;
  l.status = c.take<int32_t>(64);
  l.wmax = c.take<float>(64);
  l.dY = c.take<float>((size_t)n * dim);
  l.block_counts = c.take<int32_t>((size_t)ceil_div(e_cap > 0 ? e_cap : 1, kEdgesPerBlock) + 1);
  l.total = c.take<int64_t>(8);
  l.scan_ws = c.take<int64_t>(kScanMaxBlocks);
  l.bytes = c.bytes();
  return l;
}

static Params make_params(float a, float b, float lr, int epoch, int n_epochs) {
  Params p;
  p.a = a;
  p.b = b;
  p.m2ab = (-2.0f * a) * b;
  p.two_b = 2.0f * b;
  // the reference computes alpha in Python double and casts it to float32 (umap.py:431)
  p.alpha = (float)((double)lr * (1.0 - (double)epoch / (double)n_epochs));
  return p;
}

static unsigned edge_grid(int64_t e_cap) {
  const int64_t want = ceil_div(e_cap > 0 ? e_cap : 1, kBlock);
  const int64_t cap = (int64_t)num_sms() * 16;
  return (unsigned)(want < cap ? want : cap);
}

// a few resident blocks per SM: long warp segments keep the partial batches rare
static unsigned epoch_grid(int64_t e_cap, int blocks_per_sm) {
  const int64_t want = ceil_div(e_cap > 0 ? e_cap : 1, kBlock * 4);
  const int64_t cap = (int64_t)num_sms() * blocks_per_sm;
  return (unsigned)(want < cap ? want : cap);
}

// The kernel compiled for 5 negatives runs at that rate unless the environment sets
// UMAPB_LAYOUT_NEG5=0 (read per call): both kernels make the same draws and sums.
static bool neg5_kernel_enabled() {
  const char* e = getenv("UMAPB_LAYOUT_NEG5");
  return !(e && e[0] == '0' && e[1] == 0);
}

template <int DIM>
static void launch_epoch(const Layout& l, float* Y, int64_t n, const int32_t* rows, const int32_t* cols,
                         const float* eps, float* next, const int64_t* n_edges, int64_t e_cap, int epoch,
                         const Params& p, int neg_rate, uint64_t seed, bool neg5, cudaStream_t stream) {
  if (neg_rate == 5 && neg5)
    sgd_epoch_kernel<DIM, 5><<<epoch_grid(e_cap, kEpochBlocksPerSM5), kBlock, 0, stream>>>(
        Y, l.dY, (int)n, rows, cols, eps, next, n_edges, epoch, p, neg_rate, (uint32_t)seed, (uint32_t)(seed >> 32));
  else
    sgd_epoch_kernel<DIM, 0><<<epoch_grid(e_cap, kEpochBlocksPerSM), kBlock, 0, stream>>>(
        Y, l.dY, (int)n, rows, cols, eps, next, n_edges, epoch, p, neg_rate, (uint32_t)seed, (uint32_t)(seed >> 32));
  const int64_t m = n * DIM;
  const unsigned gb = (unsigned)(ceil_div(m, kBlock) < num_sms() * 8 ? ceil_div(m, kBlock) : num_sms() * 8);
  apply_kernel<<<gb, kBlock, 0, stream>>>(Y, l.dY, m);
}

static void launch_epoch_wide(const Layout& l, float* Y, int64_t n, int dim, const int32_t* rows,
                              const int32_t* cols, const float* eps, float* next, const int64_t* n_edges,
                              int64_t e_cap, int epoch, const Params& p, int neg_rate, uint64_t seed,
                              cudaStream_t stream) {
  const int64_t want = ceil_div(e_cap > 0 ? e_cap : 1, kBlock);
  const int64_t cap = (int64_t)num_sms() * 8;
  sgd_epoch_wide_kernel<<<(unsigned)(want < cap ? want : cap), kBlock, 0, stream>>>(
      Y, l.dY, (int)n, dim, rows, cols, eps, next, n_edges, epoch, p, neg_rate, (uint32_t)seed,
      (uint32_t)(seed >> 32));
  const int64_t m = n * dim;
  const unsigned gb = (unsigned)(ceil_div(m, kBlock) < num_sms() * 8 ? ceil_div(m, kBlock) : num_sms() * 8);
  apply_kernel<<<gb, kBlock, 0, stream>>>(Y, l.dY, m);
}

template <int DIM>
static void launch_injected(const Layout& l, float* Y, int64_t n, const int32_t* rows, const int32_t* cols,
                            const float* eps, float* next, const int64_t* n_edges, int64_t e_cap, int epoch,
                            const Params& p, int neg_rate, const int32_t* neg_to, cudaStream_t stream) {
  const unsigned nb = (unsigned)ceil_div(e_cap > 0 ? e_cap : 1, kEdgesPerBlock);
  sgd_injected_kernel<DIM><<<nb, kBlock, 0, stream>>>(Y, l.dY, rows, cols, eps, next, n_edges, epoch, p, neg_rate,
                                                      neg_to, l.block_counts, l.total);
  const int64_t m = n * DIM;
  apply_kernel<<<(unsigned)ceil_div(m, kBlock), kBlock, 0, stream>>>(Y, l.dY, m);
}

}  // namespace layout
}  // namespace umapb

using namespace umapb;

extern "C" int umapb_layout_workspace(int64_t n, int32_t dim, int64_t e_cap, size_t* bytes) {
  clear_error();
  UMAPB_REQUIRE(bytes, "bytes is null");
  UMAPB_REQUIRE(n >= 1 && dim >= 1 && dim <= 32 && e_cap >= 0, "layout: need n >= 1, 1 <= dim <= 32, e_cap >= 0");
  *bytes = layout::carve(nullptr, n, dim, e_cap).bytes;
  return UMAPB_OK;
}

extern "C" int umapb_layout_prepare(const float* vals, const int64_t* n_edges, int64_t e_cap, int32_t n_epochs,
                                    float* eps, float* next, void* workspace, size_t workspace_bytes,
                                    umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(vals && n_edges && eps && next, "layout_prepare: null array argument");
  UMAPB_REQUIRE(n_epochs >= 1, "layout_prepare: n_epochs must be >= 1");
  UMAPB_REQUIRE(workspace && workspace_bytes >= 512, "layout_prepare: workspace too small");
  layout::Layout l = layout::carve(workspace, 1, 1, 1);  // status and wmax sit at fixed offsets
  UMAPB_CUDA_TRY(cudaMemsetAsync(l.wmax, 0, 4, stream), "layout_prepare: reset");
  const unsigned g = layout::edge_grid(e_cap);
  layout::max_kernel<<<g, layout::kBlock, 0, stream>>>(vals, n_edges, l.wmax);
  layout::eps_kernel<<<g, layout::kBlock, 0, stream>>>(vals, n_edges, l.wmax, n_epochs, eps, next);
  UMAPB_LAUNCH_CHECK("layout_prepare kernels");
  count_launches(2);
  return UMAPB_OK;
}

static int enqueue_epochs(float* Y, int64_t n, int32_t dim, const int32_t* rows, const int32_t* cols,
                          const float* eps, float* next, const int64_t* n_edges, int64_t e_cap, int32_t epoch_begin,
                          int32_t epoch_end, int32_t n_epochs, float a, float b, float learning_rate,
                          int32_t neg_rate, uint64_t seed, void* workspace, size_t workspace_bytes,
                          cudaStream_t stream) {
  UMAPB_REQUIRE(Y && rows && cols && eps && next && n_edges, "layout_epochs: null array argument");
  UMAPB_REQUIRE(n >= 1 && n < ((int64_t)1 << 31), "layout_epochs: need 1 <= n < 2^31");
  UMAPB_REQUIRE(dim >= 1 && dim <= 32, "layout_epochs: dim must be in [1, 32]");
  UMAPB_REQUIRE(neg_rate >= 0, "layout_epochs: negative_sample_rate must be >= 0");
  UMAPB_REQUIRE(0 <= epoch_begin && epoch_begin <= epoch_end && epoch_end <= n_epochs,
                "layout_epochs: need 0 <= epoch_begin <= epoch_end <= n_epochs");
  layout::Layout l = layout::carve(nullptr, n, dim, e_cap);
  if (!workspace || workspace_bytes < l.bytes)
    return set_error(UMAPB_ERR_WORKSPACE, "layout: workspace of %zu bytes, need %zu", workspace_bytes, l.bytes);
  l = layout::carve(workspace, n, dim, e_cap);
  UMAPB_CUDA_TRY(cudaMemsetAsync(l.dY, 0, sizeof(float) * n * dim, stream), "layout_epochs: reset");
  const bool neg5 = layout::neg5_kernel_enabled();
  for (int ep = epoch_begin; ep < epoch_end; ++ep) {
    const layout::Params p = layout::make_params(a, b, learning_rate, ep, n_epochs);
    switch (dim) {
      case 1: layout::launch_epoch<1>(l, Y, n, rows, cols, eps, next, n_edges, e_cap, ep, p, neg_rate, seed, neg5, stream); break;
      case 2: layout::launch_epoch<2>(l, Y, n, rows, cols, eps, next, n_edges, e_cap, ep, p, neg_rate, seed, neg5, stream); break;
      case 3: layout::launch_epoch<3>(l, Y, n, rows, cols, eps, next, n_edges, e_cap, ep, p, neg_rate, seed, neg5, stream); break;
      case 4: layout::launch_epoch<4>(l, Y, n, rows, cols, eps, next, n_edges, e_cap, ep, p, neg_rate, seed, neg5, stream); break;
      default:
        layout::launch_epoch_wide(l, Y, n, dim, rows, cols, eps, next, n_edges, e_cap, ep, p, neg_rate, seed, stream);
        break;
    }
  }
  UMAPB_LAUNCH_CHECK("layout_epochs kernels");
  count_launches(2 * (epoch_end - epoch_begin));
  return UMAPB_OK;
}

extern "C" int umapb_layout_epochs(float* Y, int64_t n, int32_t dim, const int32_t* rows, const int32_t* cols,
                                   const float* eps, float* next, const int64_t* n_edges, int64_t e_cap,
                                   int32_t epoch_begin, int32_t epoch_end, int32_t n_epochs, float a, float b,
                                   float learning_rate, int32_t neg_rate, uint64_t seed, void* workspace,
                                   size_t workspace_bytes, umapb_stream_t stream_) {
  clear_error();
  return enqueue_epochs(Y, n, dim, rows, cols, eps, next, n_edges, e_cap, epoch_begin, epoch_end, n_epochs, a, b,
                        learning_rate, neg_rate, seed, workspace, workspace_bytes,
                        reinterpret_cast<cudaStream_t>(stream_));
}

// One executable graph per device, reused across calls: each call records its
// launches (stream capture, thread-local mode, on a private non-blocking stream:
// the caller's stream may be the legacy default stream, which cannot be captured),
// updates the cached executable with the new parameters (cudaGraphExecUpdate; same
// topology for the same epoch count) or instantiates a new one, and launches it on
// the caller's stream.  Updates affect later launches only, so a replay still in
// flight keeps its parameters.
namespace {
std::mutex g_graph_mu;
cudaGraphExec_t g_graph_exec[64] = {};
cudaStream_t g_capture_stream[64] = {};
}  // namespace

extern "C" int umapb_layout_epochs_graph(float* Y, int64_t n, int32_t dim, const int32_t* rows,
                                         const int32_t* cols, const float* eps, float* next, const int64_t* n_edges,
                                         int64_t e_cap, int32_t epoch_begin, int32_t epoch_end, int32_t n_epochs,
                                         float a, float b, float learning_rate, int32_t neg_rate, uint64_t seed,
                                         void* workspace, size_t workspace_bytes, umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  int dev = 0;
  UMAPB_CUDA_TRY(cudaGetDevice(&dev), "layout_epochs_graph: device");
  UMAPB_REQUIRE(dev >= 0 && dev < 64, "layout_epochs_graph: device index out of range");
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  UMAPB_CUDA_TRY(cudaStreamIsCapturing(stream, &cs), "layout_epochs_graph: capture query");
  UMAPB_REQUIRE(cs == cudaStreamCaptureStatusNone, "layout_epochs_graph: the stream is already being captured");
  std::lock_guard<std::mutex> lock(g_graph_mu);
  cudaStream_t& cap = g_capture_stream[dev];
  if (!cap) UMAPB_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "layout_epochs_graph: stream");
  UMAPB_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "layout_epochs_graph: capture");
  const int rc = enqueue_epochs(Y, n, dim, rows, cols, eps, next, n_edges, e_cap, epoch_begin, epoch_end, n_epochs, a,
                                b, learning_rate, neg_rate, seed, workspace, workspace_bytes, cap);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(cap, &graph);
  if (rc != UMAPB_OK || ce != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    if (rc != UMAPB_OK) return rc;
    return set_error(UMAPB_ERR_CUDA, "layout_epochs_graph: end of capture: %s", cudaGetErrorString(ce));
  }
  cudaGraphExec_t& exec = g_graph_exec[dev];
  if (exec) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(exec, graph, &info) != cudaSuccess) {
      cudaGetLastError();  // a topology change: instantiate anew
      cudaGraphExecDestroy(exec);
      exec = nullptr;
    }
  }
  cudaError_t e = cudaSuccess;
  if (!exec) e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    exec = nullptr;
    return set_error(UMAPB_ERR_CUDA, "layout_epochs_graph: instantiate: %s", cudaGetErrorString(e));
  }
  UMAPB_CUDA_TRY(cudaGraphLaunch(exec, stream), "layout_epochs_graph: launch");
  return UMAPB_OK;
}

extern "C" int umapb_layout_count_active(const float* next, const int64_t* n_edges, int64_t n, int32_t dim,
                                         int64_t e_cap, int32_t epoch, int64_t* count, void* workspace,
                                         size_t workspace_bytes, umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(next && n_edges && count, "layout_count_active: null array argument");
  UMAPB_REQUIRE(n >= 1 && dim >= 1 && dim <= 32, "layout_count_active: need n >= 1 and 1 <= dim <= 32");
  layout::Layout l = layout::carve(nullptr, n, dim, e_cap);
  if (!workspace || workspace_bytes < l.bytes)
    return set_error(UMAPB_ERR_WORKSPACE, "layout: workspace of %zu bytes, need %zu", workspace_bytes, l.bytes);
  l = layout::carve(workspace, n, dim, e_cap);
  const int64_t nb = ceil_div(e_cap > 0 ? e_cap : 1, layout::kEdgesPerBlock);
  layout::count_active_kernel<<<(unsigned)nb, layout::kBlock, 0, stream>>>(next, n_edges, epoch, l.block_counts);
  scan_exclusive(l.block_counts, nb, count, l.scan_ws, stream);
  UMAPB_LAUNCH_CHECK("layout_count_active kernels");
  count_launches(2);
  return UMAPB_OK;
}

extern "C" int umapb_layout_epoch_injected(float* Y, int64_t n, int32_t dim, const int32_t* rows,
                                           const int32_t* cols, const float* eps, float* next,
                                           const int64_t* n_edges, int64_t e_cap, int32_t epoch, int32_t n_epochs,
                                           float a, float b, float learning_rate, int32_t neg_rate,
                                           const int32_t* neg_to, int64_t neg_count, void* workspace,
                                           size_t workspace_bytes, umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(Y && rows && cols && eps && next && n_edges, "layout_epoch_injected: null array argument");
  UMAPB_REQUIRE(dim >= 1 && dim <= 32, "layout_epoch_injected: dim must be in [1, 32]");
  UMAPB_REQUIRE(0 <= epoch && epoch < n_epochs, "layout_epoch_injected: epoch out of range");
  UMAPB_REQUIRE(neg_rate >= 0 && neg_count >= 0, "layout_epoch_injected: negative counts must be >= 0");
  UMAPB_REQUIRE(neg_to || neg_count == 0, "layout_epoch_injected: neg_to is null");
  layout::Layout l = layout::carve(nullptr, n, dim, e_cap);
  if (!workspace || workspace_bytes < l.bytes)
    return set_error(UMAPB_ERR_WORKSPACE, "layout: workspace of %zu bytes, need %zu", workspace_bytes, l.bytes);
  l = layout::carve(workspace, n, dim, e_cap);
  UMAPB_CUDA_TRY(cudaMemsetAsync(l.dY, 0, sizeof(float) * n * dim, stream), "layout_epoch_injected: reset");
  const unsigned nb = (unsigned)ceil_div(e_cap > 0 ? e_cap : 1, layout::kEdgesPerBlock);
  layout::count_active_kernel<<<nb, layout::kBlock, 0, stream>>>(next, n_edges, epoch, l.block_counts);
  scan_exclusive(l.block_counts, (int64_t)nb, l.total, l.scan_ws, stream);
  UMAPB_LAUNCH_CHECK("layout_epoch_injected: active count");
  int64_t active = 0;
  UMAPB_CUDA_TRY(cudaMemcpyAsync(&active, l.total, sizeof(active), cudaMemcpyDeviceToHost, stream),
                 "layout_epoch_injected: count readback");
  UMAPB_CUDA_TRY(cudaStreamSynchronize(stream), "layout_epoch_injected: sync");
  if (active * neg_rate != neg_count)
    return set_error(UMAPB_ERR_ARG, "layout_epoch_injected: epoch %d has %lld active edges, so %lld negatives are "
                     "needed (got %lld)", epoch, (long long)active, (long long)(active * neg_rate),
                     (long long)neg_count);
  const layout::Params p = layout::make_params(a, b, learning_rate, epoch, n_epochs);
  switch (dim) {
    case 1: layout::launch_injected<1>(l, Y, n, rows, cols, eps, next, n_edges, e_cap, epoch, p, neg_rate, neg_to, stream); break;
    case 2: layout::launch_injected<2>(l, Y, n, rows, cols, eps, next, n_edges, e_cap, epoch, p, neg_rate, neg_to, stream); break;
    case 3: layout::launch_injected<3>(l, Y, n, rows, cols, eps, next, n_edges, e_cap, epoch, p, neg_rate, neg_to, stream); break;
    case 4: layout::launch_injected<4>(l, Y, n, rows, cols, eps, next, n_edges, e_cap, epoch, p, neg_rate, neg_to, stream); break;
    default: {
      const unsigned nb = (unsigned)ceil_div(e_cap > 0 ? e_cap : 1, layout::kEdgesPerBlock);
      layout::sgd_injected_wide_kernel<<<nb, layout::kBlock, 0, stream>>>(Y, l.dY, (int)n, dim, rows, cols, eps, next,
                                                                          n_edges, epoch, p, neg_rate, neg_to,
                                                                          l.block_counts, l.total);
      const int64_t m = n * dim;
      layout::apply_kernel<<<(unsigned)ceil_div(m, layout::kBlock), layout::kBlock, 0, stream>>>(Y, l.dY, m);
      break;
    }
  }
  UMAPB_LAUNCH_CHECK("layout_epoch_injected kernels");
  count_launches(4);
  return UMAPB_OK;
}
