// Exact brute-force kNN on B200 — replaces mlx_vis/_knn.py:47-88.
//
// 1. prep:   X (f32) -> two BF16 operands with row pitch ld = round_up(d + 3, 8):
//            A_i = [x~_i, 1, 1, 1, 0...] and B_j = [-2 x~_j, h1, h2, h3, 0...],
//            x~ = bf16(x) and h1 + h2 + h3 = |x~_j|^2 (float32 split into three
//            BF16 parts, relative error ~2^-27).  A_i . B_j is then the score
//            s_ij = |x~_j|^2 - 2 x~_i . x~_j, which orders row i's candidates by
//            distance (|x~_i|^2 is constant along the row).  The three extra K
//            columns live in padding the 64-wide K blocks carry anyway.
// 2. topk:   persistent tcgen05 kernel.  The n x n score matrix is cut into
//            tiles of 256 points (MMA N) by 256 query rows (L <= 32: a CTA pair
//            on one TPC, cluster of 2, tcgen05.mma.cta_group::2 with M = 256) or
//            by 128 rows (L > 32, or pairing switched off: one CTA, M = 128);
//            unit u (pair or CTA) owns the contiguous tile range
//            [u*T/G, (u+1)*T/G) in (row block, column tile) order.  In every CTA
//            warp 0 streams k-blocks with TMA (128-byte swizzle, zero fill past
//            n and d): its own 128 query rows and, in a pair, its half (128) of
//            the tile's points, so each CTA reads (128 + 128) x K per 128 x 256
//            outputs instead of (128 + 256) x K.  Warp 1 of the even CTA issues
//            the MMAs into one of two TMEM accumulators (2 x 256 columns, rows
//            split over the pair's TMEMs), warps 4-7 of each CTA read the
//            finished accumulator (one TMEM lane = one query row per thread) and
//            keep the row's best L scores.  When a unit leaves a row block it
//            writes the lists to cand[row][slot] (slot = which unit of that row
//            block).
// 3. rerank: one warp per row merges its slots, keeps the best L by
//            (score, index), recomputes those L distances exactly in FP32
//            (sum of (x_i - x_j)^2) and writes the k nearest by (distance, index).
// Lists of more than 128 candidates (L = k + extra > 128) go to knn_exact.cu.
#include <cuda_bf16.h>
#include <math.h>
#include <stdlib.h>

#include <mutex>
#include <vector>

#include "common.cuh"
#include "knn_exact.cuh"
#include "tc.cuh"

namespace umapb {
namespace knn {

constexpr int BM = 128;  // query rows per tile = TMEM lanes
constexpr int BN = 256;  // points per tile = MMA N
constexpr int BK = 64;   // BF16 elements per 128-byte swizzled row
constexpr int UK = 16;   // K of one tcgen05.mma kind::f16
constexpr int A_BYTES = BM * BK * 2;
constexpr int THREADS = 256;  // warp 0 TMA, warp 1 MMA, warp 2 TMEM owner, warps 4-7 epilogue

constexpr int STG_PITCH = 36;  // floats per staging row (32 scores + padding)

// LCAP == 32: each thread keeps its row's best 32 (score, column) pairs sorted in
// registers and appends hits (score below its 32nd best) to a private buffer in
// shared memory; batches of 16 are merged by data-independent sorting networks,
// so the 32 rows of a warp merge in lockstep without divergence.
// LCAP > 32: per-thread sorted lists in shared memory with insertion.
// PAIR: the CTA holds 128 of the tile's 256 points (its half of the pair's B).
template <int LCAP, bool PAIR>
struct Cfg {
  static_assert(!PAIR || LCAP == 32, "CTA pairs run the batched top-32 epilogue only");
  static constexpr bool kWarpSelect = LCAP == 32;
  static constexpr int kBBytes = (PAIR ? BN / 2 : BN) * BK * 2;
  static constexpr int kStageBytes = A_BYTES + kBBytes;
  static constexpr int kRowsPerBlock = PAIR ? 2 * BM : BM;
  static constexpr int kStages = PAIR ? 5 : (LCAP <= 64 ? 3 : 2);
  // batched selection: merge once some row of the warp holds kMergeAt hits; a
  // 32-column group then adds at most 32 to the kMergeAt - 1 already pending
  static constexpr int kMergeAt = PAIR ? 12 : 16;
  static constexpr int kBuf = kMergeAt + 32;
  static constexpr int kListBytes = kWarpSelect ? BM * kBuf * 8 + BM * STG_PITCH * 4 : BM * LCAP * 8;
  static constexpr int kBarBytes = 256;
  static constexpr int kSmem = 1024 + kStages * kStageBytes + kListBytes + kBarBytes;
};

struct Plan {
  int64_t n, d, ld;
  int64_t m, r0;  // query rows [r0, r0 + m) against all n rows (m = n, r0 = 0: every row)
  int k, L, lcap, num_kb, slots;
  bool pair;     // 256-row tiles on CTA pairs (cta_group::2)
  int rb_rows;   // query rows per row block: 256 (pair) or 128
  int64_t row_blocks, col_tiles, tiles, cols_pad;
  int64_t grid;  // work units: CTA pairs (pair) or CTAs
  size_t ws_bytes;
  // workspace layout
  int32_t* status;
  __nv_bfloat16* xa;  // A operand rows [x~, 1, 1, 1]
  __nv_bfloat16* xb;  // B operand rows [-2 x~, h1, h2, h3]
  float* cand_s;
  int32_t* cand_i;
  bool exact;       // k + extra > 128: the long-list path (knn_exact.cu)
  knnx::Plan xp;
};

__host__ __device__ inline int64_t first_cta(int64_t tile, int64_t tiles, int64_t grid) {
  // largest unit c with floor(c * tiles / grid) <= tile
  return ((tile + 1) * grid + tiles - 1) / tiles - 1;
}

// CTA pairs of the cluster launch that fit on the device at once (0: pairs
// unavailable); defined after the kernel.
static int64_t resident_pairs();

// Pairing is on unless the environment sets UMAPB_KNN_PAIR=0 (read per call).
static bool pairing_enabled() {
  const char* e = getenv("UMAPB_KNN_PAIR");
  return !(e && e[0] == '0' && e[1] == 0);
}

static int make_plan(int64_t n, int64_t d, int k, int extra, void* ws, Plan& p, int64_t r0 = 0,
                     int64_t m = -1) {
  if (m < 0) m = n;
  if (n < 2) return set_error(UMAPB_ERR_ARG, "knn_brute: need n >= 2 (got %lld)", (long long)n);
  if (r0 < 0 || m < 1 || r0 + m > n)
    return set_error(UMAPB_ERR_ARG, "knn_brute: query rows [%lld, %lld) outside [0, %lld)", (long long)r0,
                     (long long)(r0 + m), (long long)n);
  p.m = m;
  p.r0 = r0;
  if (d < 1) return set_error(UMAPB_ERR_ARG, "knn_brute: need d >= 1");
  if (k < 1 || k > n - 1) return set_error(UMAPB_ERR_ARG, "knn_brute: need 1 <= k <= n-1 (k=%d, n=%lld)", k, (long long)n);
  if (extra < 0) return set_error(UMAPB_ERR_ARG, "knn_brute: extra must be >= 0");
  if (n > (int64_t)1 << 30) return set_error(UMAPB_ERR_UNSUPPORTED, "knn_brute: n above 2^30");
  p.n = n;
  p.d = d;
  p.k = k;
  p.L = k + extra;
  if (p.L > n - 1) p.L = (int)(n - 1);
  if (p.L < k) p.L = k;
  p.exact = p.L > 128;
  if (p.exact) {  // exact distances for every pair, no candidate lists
    int s = knnx::plan(n, d, k, p.L, r0, m, ws, p.xp);
    p.ws_bytes = p.xp.bytes;
    p.status = p.xp.status;
    return s;
  }
  p.lcap = p.L <= 32 ? 32 : (p.L <= 64 ? 64 : 128);
  // features + three norm columns, padded to whole 64-element K blocks so every
  // 128-byte TMA box row starts on a 128-byte boundary
  p.ld = (d + 3 + BK - 1) / BK * BK;
  p.num_kb = (int)ceil_div(p.ld, BK);
  int64_t g = 0;
  p.pair = false;
  if (p.lcap == 32 && pairing_enabled()) {
    g = resident_pairs();
    p.pair = g > 0;
  }
  if (!p.pair) g = num_sms();
  p.rb_rows = p.pair ? 2 * BM : BM;
  p.row_blocks = ceil_div(m, p.rb_rows);
  p.col_tiles = ceil_div(n, BN);
  p.cols_pad = p.col_tiles * BN;
  p.tiles = p.row_blocks * p.col_tiles;
  p.grid = g < p.tiles ? g : p.tiles;
  int64_t slots = 1;
  for (int64_t rb = 0; rb < p.row_blocks; ++rb) {
    int64_t a = first_cta(rb * p.col_tiles, p.tiles, p.grid);
    int64_t b = first_cta(rb * p.col_tiles + p.col_tiles - 1, p.tiles, p.grid);
    if (b - a + 1 > slots) slots = b - a + 1;
  }
  p.slots = (int)slots;
  Carver c(ws);
  p.status = c.take<int32_t>(64);
  p.xa = c.take<__nv_bfloat16>((size_t)n * p.ld, 1024);
  p.xb = c.take<__nv_bfloat16>((size_t)n * p.ld, 1024);
  p.cand_s = c.take<float>((size_t)m * p.slots * p.L);
  p.cand_i = c.take<int32_t>((size_t)m * p.slots * p.L);
  p.ws_bytes = c.bytes();
  return UMAPB_OK;
}

// ---- 1. prep: augmented BF16 operands (one warp per row) ---------------------
__global__ void prep_kernel(const float* __restrict__ X, int64_t n, int d, int ld, __nv_bfloat16* __restrict__ xa,
                            __nv_bfloat16* __restrict__ xb) {
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= n) return;
  const float* xr = X + row * d;
  __nv_bfloat16* ar = xa + row * ld;
  __nv_bfloat16* br = xb + row * ld;
  float acc = 0.f;
  for (int c = lane; c < d; c += 32) {
    const __nv_bfloat16 h = __float2bfloat16_rn(__ldg(xr + c));
    const float r = __bfloat162float(h);
    ar[c] = h;
    br[c] = __float2bfloat16_rn(-2.0f * r);  // exact: a power-of-two scaling
    acc = fmaf(r, r, acc);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  // |x~|^2 = h1 + h2 + h3; each remainder is exact in float32
  const __nv_bfloat16 h1 = __float2bfloat16_rn(acc);
  const float r1 = acc - __bfloat162float(h1);
  const __nv_bfloat16 h2 = __float2bfloat16_rn(r1);
  const __nv_bfloat16 h3 = __float2bfloat16_rn(r1 - __bfloat162float(h2));
  const __nv_bfloat16 one = __float2bfloat16_rn(1.0f), zero = __float2bfloat16_rn(0.0f);
  for (int c = d + lane; c < ld; c += 32) {
    const int e = c - d;
    ar[c] = e < 3 ? one : zero;
    br[c] = e == 0 ? h1 : (e == 1 ? h2 : (e == 2 ? h3 : zero));
  }
}

// ---- sorting networks on (score, column) pairs held in registers -------------
__device__ __forceinline__ bool key_lt2(float a, int ia, float b, int ib) {
  return a < b || (a == b && ia < ib);
}

// Compare-exchange on the score alone: which of two equal scores survives at the
// 32nd slot does not change the result, because the exact rerank orders the
// surviving candidates by (distance, index).
__device__ __forceinline__ void cex(float& a, int& ia, float& b, int& ib, bool ascending) {
  const bool sw = ascending ? (b < a) : (a < b);
  const float ta = a, tb = b;
  const int xa = ia, xb = ib;
  a = sw ? tb : ta;
  b = sw ? ta : tb;
  ia = sw ? xb : xa;
  ib = sw ? xa : xb;
}

// ascending bitonic sort of 16 pairs
__device__ __forceinline__ void sort16(float (&v)[16], int (&x)[16]) {
#pragma unroll
  for (int size = 2; size <= 16; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int j = i ^ stride;
        if (j > i) cex(v[i], x[i], v[j], x[j], (i & size) == 0);
      }
    }
  }
}

// list (32, ascending) := smallest 32 of list U batch (16, ascending), ascending.
// [list, +inf x16, reversed batch] is bitonic; its half-cleaner keeps the 32
// smallest in the lower half, which a bitonic merge then sorts.
__device__ __forceinline__ void merge_32_16(float (&lv)[32], int (&li)[32], const float (&bv)[16],
                                            const int (&bx)[16]) {
#pragma unroll
  for (int i = 16; i < 32; ++i) {
    const float b = bv[31 - i];
    const int ib = bx[31 - i];
    if (b < lv[i]) {
      lv[i] = b;
      li[i] = ib;
    }
  }
#pragma unroll
  for (int stride = 16; stride > 0; stride >>= 1) {
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      if ((i & stride) == 0) cex(lv[i], li[i], lv[i + stride], li[i + stride], true);
    }
  }
}


// ---- 2. tcgen05 distance tiles + fused per-row top-L ------------------------
template <int LCAP, bool PAIR>
__global__ void __launch_bounds__(THREADS, 1)
    topk_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                int n, int num_kb, int64_t col_tiles, int64_t tiles, int slots,
                int L, float* __restrict__ cand_s, int32_t* __restrict__ cand_i, int32_t* __restrict__ status,
                int m_rows, int r0) {
  using C = Cfg<LCAP, PAIR>;
  constexpr int STAGE_BYTES = C::kStageBytes;
  constexpr int RB = C::kRowsPerBlock;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* stages = smem;
  float* list_s = reinterpret_cast<float*>(smem + C::kStages * STAGE_BYTES);  // [LCAP][BM]
  int32_t* list_i = reinterpret_cast<int32_t*>(list_s + LCAP * BM);           // [LCAP][BM]
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + C::kStages * STAGE_BYTES + C::kListBytes);
  uint64_t* full = bars;
  uint64_t* empty = bars + C::kStages;
  uint64_t* tfull = bars + 2 * C::kStages;
  uint64_t* tempty = tfull + 2;
  uint64_t* relay = tempty + 2;  // pair, rank 1: its epilogue's releases, forwarded to rank 0
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(relay + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  if constexpr (PAIR) {
    uint32_t nrank;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(nrank));
    if (nrank != 2) {  // cta_group::2 needs the cluster launch of two CTAs
      if (threadIdx.x == 0) atomicExch(status, (int32_t)kDevBadLaunch);
      return;
    }
  }
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  // rank 0 of a pair issues the MMAs and owns the full / tempty barriers the
  // pair shares; rank 1 holds accumulator rows 128-255 of each tile
  const uint32_t rank = PAIR ? tc::cluster_ctarank() : 0u;
  const int64_t G = PAIR ? (int64_t)(gridDim.x >> 1) : (int64_t)gridDim.x;
  const int64_t cta = PAIR ? (int64_t)(blockIdx.x >> 1) : (int64_t)blockIdx.x;  // work unit
  const int64_t t_begin = cta * tiles / G;
  const int64_t t_end = (cta + 1) * tiles / G;

  if (threadIdx.x == 0) {
    for (int s = 0; s < C::kStages; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      tc::mbar_init(&tfull[a], 1);
      // one arrival per epilogue thread, plus (pair) one forwarded from rank 1
      tc::mbar_init(&tempty[a], PAIR ? 129 : 128);
      tc::mbar_init(&relay[a], 128);
    }
    *abort_flag = 0;
    tc::fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    tc::prefetch_tmap(&tmA);
    tc::prefetch_tmap(&tmB);
  }
  if constexpr (PAIR) {
    // both CTAs' barriers are initialised before any remote arrival or TMA
    // completion reaches them; then the pair allocates TMEM together
    __syncthreads();
    tc::cluster_sync();
    if (warp == 2) tc::tmem_alloc_pair(tmem_slot, 512);
  } else {
    if (warp == 2) tc::tmem_alloc(tmem_slot, 512);
  }
  if (!C::kWarpSelect && warp >= 4) {
    const int r = threadIdx.x - 128;
    for (int e = 0; e < LCAP; ++e) {
      list_s[e * BM + r] = INFINITY;
      list_i[e * BM + r] = -1;
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ---------------- TMA producer (both CTAs of a pair) ----------------
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      for (int64_t t = t_begin; t < t_end; ++t) {
        const int rb = (int)(t / col_tiles);
        const int ct = (int)(t % col_tiles);
        for (int kb = 0; kb < num_kb; ++kb) {
          if (!tc::mbar_wait(&empty[stage], phase ^ 1, abort_flag)) goto producer_done;
          uint8_t* sa = stages + stage * STAGE_BYTES;
          if constexpr (PAIR) {
            // both halves complete on rank 0's full barrier, which expects the
            // bytes of both
            const uint32_t fb = tc::mapa_shared(tc::smem_u32(&full[stage]), 0);
            if (rank == 0) tc::mbar_arrive_expect_tx(&full[stage], 2 * STAGE_BYTES);
            tc::tma_load_2d_pair(sa, &tmA, fb, kb * BK, rb * RB + (int)rank * BM);
            tc::tma_load_2d_pair(sa + A_BYTES, &tmB, fb, kb * BK, ct * BN + (int)rank * (BN / 2));
          } else {
            tc::mbar_arrive_expect_tx(&full[stage], STAGE_BYTES);
            tc::tma_load_2d(sa, &tmA, &full[stage], kb * BK, rb * BM);
            tc::tma_load_2d(sa + A_BYTES, &tmB, &full[stage], kb * BK, ct * BN);
          }
          if (++stage == C::kStages) {
            stage = 0;
            phase ^= 1;
          }
        }
      }
      if constexpr (PAIR) {
        // every stage released once more: the last MMA commits have arrived on
        // this CTA's empty barriers before it may exit
        for (int i = 0; i < C::kStages; ++i) {
          if (!tc::mbar_wait(&empty[stage], phase ^ 1, abort_flag)) break;
          if (++stage == C::kStages) {
            stage = 0;
            phase ^= 1;
          }
        }
      }
    producer_done:;
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (rank 0 of a pair) ----------------
    if (lane == 0 && rank == 0) {
      constexpr uint32_t idesc = tc::idesc_bf16_f32(PAIR ? 2 * BM : BM, BN);
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      bool ok = true;
      for (int64_t t = t_begin; t < t_end; ++t) {
        if (!tc::mbar_wait(&tempty[acc], acc_phase ^ 1, abort_flag)) {
          ok = false;
          break;
        }
        tc::tc_fence_after();
        const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
        for (int kb = 0; kb < num_kb; ++kb) {
          if (!tc::mbar_wait(&full[stage], phase, abort_flag)) {
            ok = false;
            break;
          }
          tc::tc_fence_after();
          const uint32_t a_addr = tc::smem_u32(stages + stage * STAGE_BYTES);
          const uint32_t b_addr = a_addr + A_BYTES;
#pragma unroll
          for (int k = 0; k < BK / UK; ++k) {
            const uint64_t ad = tc::sw128_kmajor_desc(a_addr + k * 32);
            const uint64_t bd = tc::sw128_kmajor_desc(b_addr + k * 32);
            const uint32_t accum = (kb | k) != 0 ? 1u : 0u;
            if constexpr (PAIR)
              tc::mma_bf16_pair(d_tmem, ad, bd, idesc, accum);
            else
              tc::mma_bf16(d_tmem, ad, bd, idesc, accum);
          }
          if constexpr (PAIR)
            tc::mma_commit_pair(&empty[stage], 0x3);
          else
            tc::mma_commit(&empty[stage]);
          if (++stage == C::kStages) {
            stage = 0;
            phase ^= 1;
          }
        }
        if (!ok) break;
        if constexpr (PAIR)
          tc::mma_commit_pair(&tfull[acc], 0x3);
        else
          tc::mma_commit(&tfull[acc]);
        acc ^= 1;
        if (acc == 0) acc_phase ^= 1;
      }
      if (PAIR && ok) {
        // both accumulators released by both CTAs' epilogues: no remote arrival
        // is still on its way to this CTA when it exits
        for (int i = 0; i < 2; ++i) {
          if (!tc::mbar_wait(&tempty[acc], acc_phase ^ 1, abort_flag)) break;
          acc ^= 1;
          if (acc == 0) acc_phase ^= 1;
        }
      }
    }
  } else if (PAIR && warp == 3) {
    // ---------------- release relay (pair, rank 1) ----------------
    // Once rank 1's epilogue has drained an accumulator (128 CTA-scope arrivals
    // on relay[acc], acquired here), one cluster-scope arrival on rank 0's
    // tempty[acc] hands it back to the MMA issuer.
    if (lane == 0 && rank == 1) {
      int acc = 0;
      uint32_t acc_phase = 0;
      for (int64_t t = t_begin; t < t_end; ++t) {
        if (!tc::mbar_wait(&relay[acc], acc_phase, abort_flag)) break;
        tc::mbar_arrive_cluster(tc::mapa_shared(tc::smem_u32(&tempty[acc]), 0));
        acc ^= 1;
        if (acc == 0) acc_phase ^= 1;
      }
    }
  } else if (C::kWarpSelect && warp >= 4) {
    // ---------------- epilogue: batched per-row top-32 (L <= 32) ----------------
    // Thread r of the four epilogue warps owns TMEM lane r, i.e. query row
    // rb*128 + r.  It keeps the row's best 32 (score, column) pairs sorted in
    // registers (lv/li; lv[31] is the admission threshold) and appends every hit
    // to its own kBuf-entry buffer in shared memory (two stores, no loop).  When a
    // thread of the warp holds kMergeAt hits the whole warp merges its buffers in
    // batches of 16 with a bitonic sort network and a bitonic 32+16 merge —
    // data-independent, so the 32 rows of a warp run in lockstep.
    const int q = warp & 3;
    const int r = q * 32 + lane;
    constexpr int BUF = C::kBuf;
    float* bs = list_s;                                          // [BUF][BM]
    int32_t* bi = reinterpret_cast<int32_t*>(list_s + BUF * BM);  // [BUF][BM]
    // per-thread staging row for the chunk being appended; a pitch of 36 floats
    // keeps each quarter-warp's 16-byte stores on distinct banks
    float* stg_row = list_s + 2 * BUF * BM + r * STG_PITCH;
    float lv[32];
    int li[32];
#pragma unroll
    for (int e = 0; e < 32; ++e) {
      lv[e] = INFINITY;
      li[e] = 0x7fffffff;
    }
    int cnt = 0;
    int acc = 0;
    uint32_t acc_phase = 0;
    int64_t cur_rb = -1;
    bool ok = true;
    auto merge_pending = [&]() {
      while (__any_sync(0xffffffffu, cnt > 0)) {
        const int m = cnt < 16 ? cnt : 16;
        const int base = cnt - m;
        float bv[16];
        int bx[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          if (e < m) {
            bv[e] = bs[(base + e) * BM + r];
            bx[e] = bi[(base + e) * BM + r];
          } else {
            bv[e] = INFINITY;
            bx[e] = 0x7fffffff;
          }
        }
        cnt = base;
        sort16(bv, bx);
        merge_32_16(lv, li, bv, bx);
      }
    };
    auto flush = [&](int64_t rb) {
      merge_pending();
      const int64_t row = rb * RB + (int64_t)rank * BM + r;
      const int64_t slot = cta - first_cta(rb * col_tiles, tiles, G);
      if (row < m_rows) {
        float* cs = cand_s + (row * slots + slot) * L;
        int32_t* ci = cand_i + (row * slots + slot) * L;
#pragma unroll
        for (int e = 0; e < 32; ++e) {
          if (e < L) {
            cs[e] = lv[e];
            ci[e] = li[e] == 0x7fffffff ? -1 : li[e];
          }
        }
      }
#pragma unroll
      for (int e = 0; e < 32; ++e) {
        lv[e] = INFINITY;
        li[e] = 0x7fffffff;
      }
    };
    for (int64_t t = t_begin; t < t_end; ++t) {
      const int64_t rb = t / col_tiles;
      const int ct = (int)(t % col_tiles);
      const bool fresh = rb != cur_rb;  // warp-uniform: the lists are empty
      if (fresh) {
        if (cur_rb >= 0) flush(cur_rb);
        cur_rb = rb;
      }
      if (!tc::mbar_wait(&tfull[acc], acc_phase, abort_flag)) {
        ok = false;
        break;
      }
      tc::tc_fence_after();
      const int64_t row = rb * RB + (int64_t)rank * BM + r;
      const bool row_ok = row < m_rows;
      const int self_col = row_ok ? (int)(row + r0) : -1;
      const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * BN);
      // Admission cap of the first tile of a row block, where the empty list
      // would admit every column: per 32-column group the 4th smallest valid
      // score, maximised over the groups.  At least 4 x 8 = 32 valid scores are
      // <= that value, so the row's 32 best of the tile all are, and admitting
      // scores <= cap alone keeps the list exact while cutting the first tile's
      // hits from 256 to about the best fifth.  A group with fewer than 4 valid
      // columns leaves the cap infinite.
      float cap = INFINITY;
      if (fresh) {
        float hi = -INFINITY;
#pragma unroll 1
        for (int ch = 0; ch < BN / 32; ++ch) {
          float v[32];
          __syncwarp();
          tc::tmem_ld32(taddr + ch * 32, v);
          const int col0 = ct * BN + ch * 32;
          float a0 = INFINITY, a1 = INFINITY, a2 = INFINITY, a3 = INFINITY;  // 4 smallest, sorted
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int col = col0 + j;
            const float x = (col != self_col && col < n) ? v[j] : INFINITY;
            a3 = fminf(a3, fmaxf(a2, x));
            a2 = fminf(a2, fmaxf(a1, x));
            a1 = fminf(a1, fmaxf(a0, x));
            a0 = fminf(a0, x);
          }
          hi = fmaxf(hi, a3);
        }
        // v <= hi  <=>  v < next float above hi (hi finite); infinite hi admits all
        cap = hi < INFINITY ? nextafterf(hi, INFINITY) : INFINITY;
      }
#pragma unroll 1
      for (int ch = 0; ch < BN / 32; ++ch) {
        float v[32];
        __syncwarp();
        tc::tmem_ld32(taddr + ch * 32, v);
        const int col0 = ct * BN + ch * 32;
        // branch-free hit mask of the 32 columns (four independent OR chains);
        // rows past n never admit
        const float tau = row_ok ? fminf(lv[31], cap) : -INFINITY;
        unsigned m0 = 0, m1 = 0, m2 = 0, m3 = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          m0 |= (v[j] < tau ? 1u : 0u) << j;
          m1 |= (v[j + 8] < tau ? 1u : 0u) << j;
          m2 |= (v[j + 16] < tau ? 1u : 0u) << j;
          m3 |= (v[j + 24] < tau ? 1u : 0u) << j;
        }
        unsigned mask = m0 | (m1 << 8) | (m2 << 16) | (m3 << 24);
        const int self_off = self_col - col0;  // the row itself
        if ((unsigned)self_off < 32u) mask &= ~(1u << self_off);
        const int lim = n - col0;  // zero-filled columns past n
        if (lim < 32) mask &= lim <= 0 ? 0u : ((1u << lim) - 1u);
        if (mask) {  // stage the chunk, then append the hits in column order
          float4* st4 = reinterpret_cast<float4*>(stg_row);
#pragma unroll
          for (int j4 = 0; j4 < 8; ++j4) st4[j4] = make_float4(v[4 * j4], v[4 * j4 + 1], v[4 * j4 + 2], v[4 * j4 + 3]);
          while (mask) {
            const int j = __ffs(mask) - 1;
            mask &= mask - 1u;
            bs[cnt * BM + r] = stg_row[j];
            bi[cnt * BM + r] = col0 + j;
            ++cnt;
          }
        }
        if (__any_sync(0xffffffffu, cnt >= C::kMergeAt)) merge_pending();
      }
      tc::tc_fence_before();
      // CTA-scope arrivals only: a cluster-scope release costs each epilogue
      // warp over a thousand cycles per tile, so rank 1's warp 3 forwards them
      tc::mbar_arrive(PAIR && rank == 1 ? &relay[acc] : &tempty[acc]);
      acc ^= 1;
      if (acc == 0) acc_phase ^= 1;
    }
    if (ok && cur_rb >= 0) flush(cur_rb);
  } else if (!C::kWarpSelect && warp >= 4) {
    // ---------------- epilogue: per-row top-L ----------------
    const int q = warp & 3;  // TMEM lane quarter of this warp
    const int r = q * 32 + lane;
    float tau = INFINITY;
    int acc = 0;
    uint32_t acc_phase = 0;
    int64_t cur_rb = -1;
    bool ok = true;
    auto flush = [&](int64_t rb) {
      const int64_t row = rb * BM + r;
      const int64_t slot = cta - first_cta(rb * col_tiles, tiles, G);
      if (row < m_rows) {
        float* cs = cand_s + (row * slots + slot) * L;
        int32_t* ci = cand_i + (row * slots + slot) * L;
        for (int e = 0; e < L; ++e) {
          cs[e] = list_s[e * BM + r];
          ci[e] = list_i[e * BM + r];
        }
      }
      for (int e = 0; e < LCAP; ++e) {
        list_s[e * BM + r] = INFINITY;
        list_i[e * BM + r] = -1;
      }
    };
    for (int64_t t = t_begin; t < t_end; ++t) {
      const int64_t rb = t / col_tiles;
      const int ct = (int)(t % col_tiles);
      if (rb != cur_rb) {
        if (cur_rb >= 0) flush(cur_rb);
        cur_rb = rb;
        tau = INFINITY;
      }
      if (!tc::mbar_wait(&tfull[acc], acc_phase, abort_flag)) {
        ok = false;
        break;
      }
      tc::tc_fence_after();
      const int64_t row = rb * BM + r;
      const bool row_ok = row < m_rows;
      const int self_col = (int)(row + r0);
      const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * BN);
#pragma unroll 1
      for (int ch = 0; ch < BN / 32; ++ch) {
        float v[32];
        __syncwarp();
        tc::tmem_ld32(taddr + ch * 32, v);
        const int col0 = ct * BN + ch * 32;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const float s = v[j];
          const int col = col0 + j;
          if (s < tau && row_ok && col != self_col && col < n) {
            int p = L - 1;
            while (p > 0) {
              const float prev = list_s[(p - 1) * BM + r];
              if (prev <= s) break;
              list_s[p * BM + r] = prev;
              list_i[p * BM + r] = list_i[(p - 1) * BM + r];
              --p;
            }
            list_s[p * BM + r] = s;
            list_i[p * BM + r] = col;
            tau = list_s[(L - 1) * BM + r];
          }
        }
      }
      tc::tc_fence_before();
      tc::mbar_arrive(&tempty[acc]);
      acc ^= 1;
      if (acc == 0) acc_phase ^= 1;
    }
    if (ok && cur_rb >= 0) flush(cur_rb);
  }

  tc::tc_fence_before();
  __syncthreads();
  if constexpr (PAIR) {
    // neither CTA frees the pair's TMEM or leaves while the other still works
    tc::cluster_sync();
    if (warp == 2) {
      tc::tc_fence_after();
      tc::tmem_dealloc_pair(tmem_base, 512);
    }
  } else if (warp == 2) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem_base, 512);
  }
  if (threadIdx.x == 0 && *abort_flag) atomicExch(status, (int32_t)kDevTimeoutEpilogue);
}

// ---- 3. merge slots + exact FP32 rerank -------------------------------------
__device__ __forceinline__ bool key_less(float a, int ia, float b, int ib) {
  return a < b || (a == b && (unsigned)ia < (unsigned)ib);
}

// Warp-cooperative bitonic sort of P (power of two) (key, idx) pairs in shared memory.
__device__ void warp_bitonic(float* key, int* idx, int P, int lane) {
  for (int size = 2; size <= P; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = lane; i < (P >> 1); i += 32) {
        const int lo = 2 * i - (i & (stride - 1));
        const int hi = lo + stride;
        const bool asc = (lo & size) == 0;
        const float ka = key[lo], kb = key[hi];
        const int ia = idx[lo], ib = idx[hi];
        const bool swap = asc ? key_less(kb, ib, ka, ia) : key_less(ka, ia, kb, ib);
        if (swap) {
          key[lo] = kb;
          key[hi] = ka;
          idx[lo] = ib;
          idx[hi] = ia;
        }
      }
      __syncwarp();
    }
  }
}

constexpr int RR_WARPS = 8;

__global__ void __launch_bounds__(RR_WARPS * 32)
    rerank_kernel(const float* __restrict__ X, int64_t n, int d, const float* __restrict__ cand_s,
                  const int32_t* __restrict__ cand_i, int slots, int L, int P, int PL, int k, int squared,
                  int32_t* __restrict__ out_idx, float* __restrict__ out_dist, int64_t r0 = 0) {
  extern __shared__ uint8_t smem_raw[];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  float* key = reinterpret_cast<float*>(smem_raw) + (size_t)warp * 2 * P;
  int* idx = reinterpret_cast<int*>(key + P);
  const int64_t row = (int64_t)blockIdx.x * RR_WARPS + warp;
  if (row >= n) return;
  const int m = slots * L;
  for (int e = lane; e < P; e += 32) {
    float s = INFINITY;
    int j = 0x7fffffff;
    if (e < m) {
      const int c = cand_i[row * m + e];
      if (c >= 0) {
        s = cand_s[row * m + e];
        j = c;
      }
    }
    key[e] = s;
    idx[e] = j;
  }
  __syncwarp();
  warp_bitonic(key, idx, P, lane);
  // exact squared distances of the best L candidates (direct form, FP32), four
  // candidates per pass so every lane keeps several independent loads in flight
  const float* xr = X + (r0 + row) * d;  // rows: the query range [r0, r0 + n)
  const bool vec = (d & 3) == 0 && (reinterpret_cast<uintptr_t>(X) & 15) == 0;
  for (int e0 = 0; e0 < PL; e0 += 4) {
    int j[4];
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int u = 0; u < 4; ++u) j[u] = (e0 + u < L) ? idx[e0 + u] : 0x7fffffff;
    if (vec) {
      const float4* xr4 = reinterpret_cast<const float4*>(xr);
      for (int c = lane; c < (d >> 2); c += 32) {
        const float4 a = __ldg(xr4 + c);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (j[u] != 0x7fffffff) {
            const float4 b = __ldg(reinterpret_cast<const float4*>(X + (int64_t)j[u] * d) + c);
            const float t0 = a.x - b.x, t1 = a.y - b.y, t2 = a.z - b.z, t3 = a.w - b.w;
            acc[u] = fmaf(t0, t0, acc[u]);
            acc[u] = fmaf(t1, t1, acc[u]);
            acc[u] = fmaf(t2, t2, acc[u]);
            acc[u] = fmaf(t3, t3, acc[u]);
          }
        }
      }
    } else {
      for (int c = lane; c < d; c += 32) {
        const float a = __ldg(xr + c);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (j[u] != 0x7fffffff) {
            const float t = a - __ldg(X + (int64_t)j[u] * d + c);
            acc[u] = fmaf(t, t, acc[u]);
          }
        }
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc[u] += __shfl_xor_sync(0xffffffffu, acc[u], o);
    }
    __syncwarp();
    if (lane < 4 && e0 + lane < PL) {
      float a = acc[0];
      int jj = j[0];
#pragma unroll
      for (int u = 1; u < 4; ++u)
        if (lane == u) {
          a = acc[u];
          jj = j[u];
        }
      key[e0 + lane] = jj != 0x7fffffff ? a : INFINITY;
      idx[e0 + lane] = jj;
    }
    __syncwarp();
  }
  warp_bitonic(key, idx, PL, lane);
  for (int e = lane; e < k; e += 32) {
    const float v = key[e];
    out_idx[row * k + e] = idx[e];
    out_dist[row * k + e] = squared ? v : sqrtf(v);
  }
}

template <int LCAP, bool PAIR>
static int set_smem_attr() {
  using C = Cfg<LCAP, PAIR>;
  static bool attr_set[64] = {false};
  int dev = 0;
  UMAPB_CUDA_TRY(cudaGetDevice(&dev), "knn_brute: cudaGetDevice");
  if (dev < 0 || dev >= 64) return set_error(UMAPB_ERR_UNSUPPORTED, "knn_brute: device index %d", dev);
  if (!attr_set[dev]) {
    UMAPB_CUDA_TRY(cudaFuncSetAttribute(topk_kernel<LCAP, PAIR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        C::kSmem),
                   "knn_brute: set smem attribute");
    attr_set[dev] = true;
  }
  return UMAPB_OK;
}

// The rerank kernel's dynamic shared memory (2 P floats per warp) can exceed the
// 48 KB default; the attribute is raised once per device (up to 200 KB).
static int rerank_smem_attr(size_t smem) {
  if (smem <= 48 * 1024) return UMAPB_OK;
  if (smem > 200 * 1024)
    return set_error(UMAPB_ERR_UNSUPPORTED, "knn_brute: candidate merge needs %zu bytes of shared memory", smem);
  static std::mutex mu;
  static bool done[64] = {false};
  int dev = 0;
  UMAPB_CUDA_TRY(cudaGetDevice(&dev), "knn_brute: cudaGetDevice");
  if (dev < 0 || dev >= 64) return set_error(UMAPB_ERR_UNSUPPORTED, "knn_brute: device index %d", dev);
  std::lock_guard<std::mutex> lock(mu);
  if (!done[dev]) {
    UMAPB_CUDA_TRY(cudaFuncSetAttribute(rerank_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(200 * 1024)),
                   "knn_brute: rerank smem attribute");
    done[dev] = true;
  }
  return UMAPB_OK;
}

static int64_t resident_pairs() {
  static std::mutex mu;
  static int64_t cached[64];
  static bool known[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
  std::lock_guard<std::mutex> lock(mu);
  if (!known[dev]) {
    int64_t pairs = 0;
    if (set_smem_attr<32, true>() == UMAPB_OK) {
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = 2;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3(2 * (unsigned)num_sms(), 1, 1);
      cfg.blockDim = dim3(THREADS, 1, 1);
      cfg.dynamicSmemBytes = Cfg<32, true>::kSmem;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int clusters = 0;
      if (cudaOccupancyMaxActiveClusters(&clusters, topk_kernel<32, true>, &cfg) == cudaSuccess) pairs = clusters;
    }
    cudaGetLastError();  // a refused query only disables pairing
    clear_error();
    cached[dev] = pairs;
    known[dev] = true;
  }
  return cached[dev];
}

template <int LCAP>
static int launch_topk(const Plan& p, const CUtensorMap& ta, const CUtensorMap& tb, cudaStream_t stream) {
  int s = set_smem_attr<LCAP, false>();
  if (s) return s;
  topk_kernel<LCAP, false><<<(unsigned)p.grid, THREADS, Cfg<LCAP, false>::kSmem, stream>>>(
      ta, tb, (int)p.n, p.num_kb, p.col_tiles, p.tiles, p.slots, p.L, p.cand_s, p.cand_i, p.status, (int)p.m,
      (int)p.r0);
  UMAPB_LAUNCH_CHECK("knn_brute: topk kernel launch");
  return UMAPB_OK;
}

static int launch_topk_pair(const Plan& p, const CUtensorMap& ta, const CUtensorMap& tb, cudaStream_t stream) {
  int s = set_smem_attr<32, true>();
  if (s) return s;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(2 * (unsigned)p.grid, 1, 1);
  cfg.blockDim = dim3(THREADS, 1, 1);
  cfg.dynamicSmemBytes = Cfg<32, true>::kSmem;
  cfg.stream = stream;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  UMAPB_CUDA_TRY(cudaLaunchKernelEx(&cfg, topk_kernel<32, true>, ta, tb, (int)p.n, p.num_kb, p.col_tiles, p.tiles,
                                    p.slots, p.L, p.cand_s, p.cand_i, p.status, (int)p.m, (int)p.r0),
                 "knn_brute: pair topk kernel launch");
  return UMAPB_OK;
}

// Tensor maps of both operands (B box: the CTA's share of a 256-point tile) and
// the tile kernel the plan chose.
static int run_tiles(const Plan& p, cudaStream_t stream) {
  CUtensorMap ta, tb;
  int s;
  if ((s = make_tmap_bf16_2d(&ta, p.xa + p.r0 * p.ld, (uint64_t)p.m, (uint64_t)p.ld, (uint64_t)p.ld, BM, BK)))
    return s;
  if ((s = make_tmap_bf16_2d(&tb, p.xb, (uint64_t)p.n, (uint64_t)p.ld, (uint64_t)p.ld, p.pair ? BN / 2 : BN, BK)))
    return s;
  if (p.pair) return launch_topk_pair(p, ta, tb, stream);
  if (p.lcap == 32) return launch_topk<32>(p, ta, tb, stream);
  if (p.lcap == 64) return launch_topk<64>(p, ta, tb, stream);
  return launch_topk<128>(p, ta, tb, stream);
}

static int next_pow2(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}

}  // namespace knn
}  // namespace umapb

using namespace umapb;

extern "C" int umapb_knn_brute_workspace(int64_t n, int64_t d, int32_t k, int32_t extra, size_t* bytes) {
  clear_error();
  if (!bytes) return set_error(UMAPB_ERR_ARG, "bytes is null");
  knn::Plan p;
  int s = knn::make_plan(n, d, k, extra, nullptr, p);
  if (s) return s;
  *bytes = p.ws_bytes;
  return UMAPB_OK;
}

// The three stages of one call; with `ev` (4 events) each stage boundary is recorded.
static int enqueue_knn(const float* X, int64_t n, int64_t d, int32_t k, int32_t squared, int32_t* out_idx,
                       float* out_dist, const knn::Plan& p, cudaStream_t stream, cudaEvent_t* ev) {
  if (p.exact) {
    if (ev) return set_error(UMAPB_ERR_UNSUPPORTED, "knn_brute_timed: k + extra must be <= 128");
    return knnx::run(X, p.xp, squared, out_idx, out_dist, stream);
  }
  int s;
  const int P = knn::next_pow2(p.slots * p.L);
  const int PL = knn::next_pow2(p.L);
  const size_t smem = (size_t)knn::RR_WARPS * 2 * P * sizeof(float);
  if ((s = knn::rerank_smem_attr(smem))) return s;
  UMAPB_CUDA_TRY(cudaMemsetAsync(p.status, 0, sizeof(int32_t), stream), "knn_brute: status reset");
  UMAPB_CUDA_TRY(cudaMemsetAsync(p.cand_i, 0xFF, (size_t)p.m * p.slots * p.L * sizeof(int32_t), stream),
                 "knn_brute: candidate reset");
  if (ev) UMAPB_CUDA_TRY(cudaEventRecord(ev[0], stream), "knn_brute: event");
  {
    const int64_t warps = n;
    const unsigned blocks = (unsigned)ceil_div(warps * 32, 256);
    knn::prep_kernel<<<blocks, 256, 0, stream>>>(X, n, (int)d, (int)p.ld, p.xa, p.xb);
    UMAPB_LAUNCH_CHECK("knn_brute: prep kernel launch");
  }
  if (ev) UMAPB_CUDA_TRY(cudaEventRecord(ev[1], stream), "knn_brute: event");
  if ((s = knn::run_tiles(p, stream))) return s;
  if (ev) UMAPB_CUDA_TRY(cudaEventRecord(ev[2], stream), "knn_brute: event");
  {
    const unsigned blocks = (unsigned)ceil_div(p.m, knn::RR_WARPS);
    knn::rerank_kernel<<<blocks, knn::RR_WARPS * 32, smem, stream>>>(X, p.m, (int)d, p.cand_s, p.cand_i, p.slots,
                                                                      p.L, P, PL, k, squared, out_idx, out_dist,
                                                                      p.r0);
    UMAPB_LAUNCH_CHECK("knn_brute: rerank kernel launch");
  }
  if (ev) UMAPB_CUDA_TRY(cudaEventRecord(ev[3], stream), "knn_brute: event");
  count_launches(3);
  return UMAPB_OK;
}

extern "C" int umapb_knn_brute(const float* X, int64_t n, int64_t d, int32_t k, int32_t extra, int32_t squared,
                               int32_t* out_idx, float* out_dist, void* workspace, size_t workspace_bytes,
                               umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(X && out_idx && out_dist, "knn_brute: null array argument");
  knn::Plan p;
  int s = knn::make_plan(n, d, k, extra, nullptr, p);
  if (s) return s;
  if (!workspace || workspace_bytes < p.ws_bytes)
    return set_error(UMAPB_ERR_WORKSPACE, "knn_brute: workspace of %zu bytes, need %zu", workspace_bytes, p.ws_bytes);
  knn::make_plan(n, d, k, extra, workspace, p);
  return enqueue_knn(X, n, d, k, squared, out_idx, out_dist, p, stream, nullptr);
}

extern "C" int umapb_knn_brute_rows_workspace(int64_t n, int64_t d, int32_t k, int32_t extra, int64_t row_begin,
                                              int64_t row_count, size_t* bytes) {
  clear_error();
  if (!bytes) return set_error(UMAPB_ERR_ARG, "bytes is null");
  knn::Plan p;
  int s = knn::make_plan(n, d, k, extra, nullptr, p, row_begin, row_count);
  if (s) return s;
  *bytes = p.ws_bytes;
  return UMAPB_OK;
}

extern "C" int umapb_knn_brute_rows(const float* X, int64_t n, int64_t d, int32_t k, int32_t extra, int32_t squared,
                                    int64_t row_begin, int64_t row_count, int32_t* out_idx, float* out_dist,
                                    void* workspace, size_t workspace_bytes, umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(X && out_idx && out_dist, "knn_brute_rows: null array argument");
  knn::Plan p;
  int s = knn::make_plan(n, d, k, extra, nullptr, p, row_begin, row_count);
  if (s) return s;
  if (!workspace || workspace_bytes < p.ws_bytes)
    return set_error(UMAPB_ERR_WORKSPACE, "knn_brute_rows: workspace of %zu bytes, need %zu", workspace_bytes,
                     p.ws_bytes);
  knn::make_plan(n, d, k, extra, workspace, p, row_begin, row_count);
  return enqueue_knn(X, n, d, k, squared, out_idx, out_dist, p, stream, nullptr);
}

extern "C" int umapb_knn_brute_timed(const float* X, int64_t n, int64_t d, int32_t k, int32_t extra, int32_t squared,
                                     int32_t* out_idx, float* out_dist, void* workspace, size_t workspace_bytes,
                                     float* stage_ms, umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(X && out_idx && out_dist && stage_ms, "knn_brute_timed: null argument");
  knn::Plan p;
  int s = knn::make_plan(n, d, k, extra, nullptr, p);
  if (s) return s;
  if (!workspace || workspace_bytes < p.ws_bytes)
    return set_error(UMAPB_ERR_WORKSPACE, "knn_brute: workspace of %zu bytes, need %zu", workspace_bytes, p.ws_bytes);
  knn::make_plan(n, d, k, extra, workspace, p);
  cudaEvent_t ev[4] = {};
  for (int i = 0; i < 4; ++i) UMAPB_CUDA_TRY(cudaEventCreate(&ev[i]), "knn_brute_timed: event create");
  s = enqueue_knn(X, n, d, k, squared, out_idx, out_dist, p, stream, ev);
  if (s == UMAPB_OK) {
    cudaError_t e = cudaEventSynchronize(ev[3]);
    for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = cudaEventElapsedTime(&stage_ms[i], ev[i], ev[i + 1]);
    if (e != cudaSuccess) s = set_error(UMAPB_ERR_CUDA, "knn_brute_timed: %s", cudaGetErrorString(e));
  }
  for (int i = 0; i < 4; ++i) cudaEventDestroy(ev[i]);
  return s;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of umapb_knn_brute.
//
// Some callers cannot hand this library a device workspace: cudaMalloc and
// cudaFree synchronise the whole device (a stall that latency-bound callers
// cannot take), they fail outright when another framework's pooled allocator
// already owns the device memory, and thin FFI bindings often have no way to
// keep a device buffer alive between calls.  This entry point therefore uses a
// fixed scratch array that lives in the library itself: a file-scope
// __device__ array of UMAPB_NOALLOC_SCRATCH_BYTES, which every GPU that loads
// the library holds until the process exits.  Requests whose workspace would
// exceed it are rejected.  The first call on each device looks up that
// device's address of the array with cudaGetSymbolAddress (with the device
// current); make that first call before any stream capture begins.  All calls
// share the one array and it keeps the previous call's contents, so the parts
// that must start at zero (the status word and the candidate lists) are reset
// by each call, and calls whose work overlaps on the GPU (for example on two
// streams at once) race on it: serialise them.
// ---------------------------------------------------------------------------
namespace {

static __device__ __align__(256) unsigned char g_knn_scratch[UMAPB_NOALLOC_SCRATCH_BYTES];

std::mutex g_scratch_mu;
void* g_scratch_addr[64] = {nullptr};

int scratch_address(void** out) {
  int dev = 0;
  UMAPB_CUDA_TRY(cudaGetDevice(&dev), "knn_brute_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= 64) return set_error(UMAPB_ERR_UNSUPPORTED, "knn_brute_noalloc: device index %d", dev);
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_knn_scratch);
    if (e != cudaSuccess)
      return set_error(UMAPB_ERR_CUDA, "knn_brute_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return UMAPB_OK;
}

}  // namespace

extern "C" int umapb_knn_brute_noalloc(const float* X, int64_t n, int64_t d, int32_t k, int32_t extra,
                                       int32_t squared, int32_t* out_idx, float* out_dist, int32_t* device_status,
                                       umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(X && out_idx && out_dist, "knn_brute_noalloc: null array argument");
  knn::Plan p;
  int s = knn::make_plan(n, d, k, extra, nullptr, p);
  if (s) return s;
  if (p.ws_bytes > (size_t)UMAPB_NOALLOC_SCRATCH_BYTES)
    return set_error(UMAPB_ERR_UNSUPPORTED,
                     "knn_brute_noalloc: n=%lld, d=%lld, k+extra=%d needs %zu bytes of scratch but the static array "
                     "holds %zu; use umapb_knn_brute with a caller-owned workspace",
                     (long long)n, (long long)d, p.L, p.ws_bytes, (size_t)UMAPB_NOALLOC_SCRATCH_BYTES);
  void* scratch = nullptr;
  if ((s = scratch_address(&scratch))) return s;
  knn::make_plan(n, d, k, extra, scratch, p);
  if (p.exact) {
    if ((s = knnx::run(X, p.xp, squared, out_idx, out_dist, stream))) return s;
    if (device_status)
      UMAPB_CUDA_TRY(cudaMemcpyAsync(device_status, p.status, sizeof(int32_t), cudaMemcpyDeviceToDevice, stream),
                     "knn_brute_noalloc: status copy");
    return UMAPB_OK;
  }

  const int P = knn::next_pow2(p.slots * p.L);
  const int PL = knn::next_pow2(p.L);
  const size_t smem = (size_t)knn::RR_WARPS * 2 * P * sizeof(float);
  if ((s = knn::rerank_smem_attr(smem))) return s;  // before any launch: a refusal leaves nothing enqueued

  UMAPB_CUDA_TRY(cudaMemsetAsync(p.status, 0, sizeof(int32_t), stream), "knn_brute_noalloc: status reset");
  UMAPB_CUDA_TRY(cudaMemsetAsync(p.cand_i, 0xFF, (size_t)n * p.slots * p.L * sizeof(int32_t), stream),
                 "knn_brute_noalloc: candidate reset");
  knn::prep_kernel<<<(unsigned)ceil_div(n * 32, 256), 256, 0, stream>>>(X, n, (int)d, (int)p.ld, p.xa, p.xb);
  UMAPB_LAUNCH_CHECK("knn_brute_noalloc: prep kernel launch");
  if ((s = knn::run_tiles(p, stream))) return s;
  knn::rerank_kernel<<<(unsigned)ceil_div(n, knn::RR_WARPS), knn::RR_WARPS * 32, smem, stream>>>(
      X, n, (int)d, p.cand_s, p.cand_i, p.slots, p.L, P, PL, k, squared, out_idx, out_dist);
  UMAPB_LAUNCH_CHECK("knn_brute_noalloc: rerank kernel launch");
  if (device_status)
    UMAPB_CUDA_TRY(cudaMemcpyAsync(device_status, p.status, sizeof(int32_t), cudaMemcpyDeviceToDevice, stream),
                   "knn_brute_noalloc: status copy");
  count_launches(3);
  return UMAPB_OK;
}
