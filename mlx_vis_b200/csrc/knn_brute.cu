// Exact brute-force kNN on B200 — replaces mlx_vis/_knn.py:47-88.
//
// 1. prep:   X (f32) -> Xb (bf16, row pitch ld = round_up(d, 8)) and
//            sqb[j] = |bf16(x_j)|^2 (f32); sqb = +inf for padded columns.
// 2. topk:   persistent tcgen05 kernel.  The n x n score matrix is cut into
//            128 x 256 tiles (query rows x points); CTA c owns the contiguous
//            tile range [c*T/G, (c+1)*T/G) in (row block, column tile) order.
//            warp 0 streams A/B k-blocks with TMA (128-byte swizzle, zero fill
//            past n and d), warp 1 issues tcgen05.mma into one of two TMEM
//            accumulators (2 x 256 columns), warps 4-7 read the finished
//            accumulator (one TMEM lane = one query row per thread) and keep
//            the row's best L scores s_j = sqb_j - 2 x_i.x_j in a sorted list in
//            shared memory.  When the CTA leaves a row block it writes the lists
//            to cand[row][slot] (slot = which CTA of that row block).
// 3. rerank: one warp per row merges its slots, keeps the best L by
//            (score, index), recomputes those L distances exactly in FP32
//            (sum of (x_i - x_j)^2) and writes the k nearest by (distance, index).
#include <cuda_bf16.h>
#include <math.h>

#include <vector>

#include "common.cuh"
#include "tc.cuh"

namespace umapb {
namespace knn {

constexpr int BM = 128;  // query rows per tile = TMEM lanes
constexpr int BN = 256;  // points per tile = MMA N
constexpr int BK = 64;   // BF16 elements per 128-byte swizzled row
constexpr int UK = 16;   // K of one tcgen05.mma kind::f16
constexpr int A_BYTES = BM * BK * 2;
constexpr int B_BYTES = BN * BK * 2;
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int THREADS = 256;  // warp 0 TMA, warp 1 MMA, warp 2 TMEM owner, warps 4-7 epilogue

template <int LCAP>
struct Cfg {
  static constexpr int kStages = LCAP <= 32 ? 4 : (LCAP <= 64 ? 3 : 2);
  static constexpr int kListBytes = BM * LCAP * 8;
  static constexpr int kBarBytes = 256;
  static constexpr int kSmem = 1024 + kStages * STAGE_BYTES + kListBytes + kBarBytes;
};

struct Plan {
  int64_t n, d, ld;
  int k, L, lcap, num_kb, slots;
  int64_t row_blocks, col_tiles, tiles, grid, cols_pad;
  size_t ws_bytes;
  // workspace layout
  int32_t* status;
  __nv_bfloat16* xb;
  float* sqb;
  float* cand_s;
  int32_t* cand_i;
};

__host__ __device__ inline int64_t first_cta(int64_t tile, int64_t tiles, int64_t grid) {
  // largest c with floor(c * tiles / grid) <= tile
  return ((tile + 1) * grid + tiles - 1) / tiles - 1;
}

static int make_plan(int64_t n, int64_t d, int k, int extra, void* ws, Plan& p) {
  if (n < 2) return set_error(UMAPB_ERR_ARG, "knn_brute: need n >= 2 (got %lld)", (long long)n);
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
  if (p.L > 128) return set_error(UMAPB_ERR_UNSUPPORTED, "knn_brute: k + extra must be <= 128 (got %d)", k + extra);
  p.lcap = p.L <= 32 ? 32 : (p.L <= 64 ? 64 : 128);
  p.ld = (d + 7) / 8 * 8;
  p.num_kb = (int)ceil_div(p.ld, BK);
  p.row_blocks = ceil_div(n, BM);
  p.col_tiles = ceil_div(n, BN);
  p.cols_pad = p.col_tiles * BN;
  p.tiles = p.row_blocks * p.col_tiles;
  int64_t g = num_sms();
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
  p.xb = c.take<__nv_bfloat16>((size_t)n * p.ld, 1024);
  p.sqb = c.take<float>((size_t)p.cols_pad);
  p.cand_s = c.take<float>((size_t)n * p.slots * p.L);
  p.cand_i = c.take<int32_t>((size_t)n * p.slots * p.L);
  p.ws_bytes = c.bytes();
  return UMAPB_OK;
}

// ---- 1. prep: bf16 copy + norms of the rounded rows -------------------------
__global__ void prep_kernel(const float* __restrict__ X, int64_t n, int d, int ld, __nv_bfloat16* __restrict__ xb,
                            float* __restrict__ sqb, int64_t cols_pad) {
  const int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= cols_pad) return;
  if (row >= n) {
    if (lane == 0) sqb[row] = INFINITY;
    return;
  }
  const float* xr = X + row * d;
  __nv_bfloat16* br = xb + row * ld;
  float acc = 0.f;
  for (int c = lane; c < ld; c += 32) {
    const float v = c < d ? __ldg(xr + c) : 0.f;
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    br[c] = h;
    const float r = __bfloat162float(h);
    acc = fmaf(r, r, acc);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) sqb[row] = acc;
}

// ---- 2. tcgen05 distance tiles + fused per-row top-L ------------------------
template <int LCAP>
__global__ void __launch_bounds__(THREADS, 1)
    topk_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                const float* __restrict__ sqb, int n, int num_kb, int64_t col_tiles, int64_t tiles, int slots,
                int L, float* __restrict__ cand_s, int32_t* __restrict__ cand_i, int32_t* __restrict__ status) {
  using C = Cfg<LCAP>;
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
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t G = gridDim.x;
  const int64_t cta = blockIdx.x;
  const int64_t t_begin = cta * tiles / G;
  const int64_t t_end = (cta + 1) * tiles / G;

  if (threadIdx.x == 0) {
    for (int s = 0; s < C::kStages; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      tc::mbar_init(&tfull[a], 1);
      tc::mbar_init(&tempty[a], 128);
    }
    *abort_flag = 0;
    tc::fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    tc::prefetch_tmap(&tmA);
    tc::prefetch_tmap(&tmB);
  }
  if (warp == 2) tc::tmem_alloc(tmem_slot, 512);
  if (warp >= 4) {
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
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      for (int64_t t = t_begin; t < t_end; ++t) {
        const int rb = (int)(t / col_tiles);
        const int ct = (int)(t % col_tiles);
        for (int kb = 0; kb < num_kb; ++kb) {
          if (!tc::mbar_wait(&empty[stage], phase ^ 1, abort_flag)) goto producer_done;
          uint8_t* sa = stages + stage * STAGE_BYTES;
          tc::mbar_arrive_expect_tx(&full[stage], STAGE_BYTES);
          tc::tma_load_2d(sa, &tmA, &full[stage], kb * BK, rb * BM);
          tc::tma_load_2d(sa + A_BYTES, &tmB, &full[stage], kb * BK, ct * BN);
          if (++stage == C::kStages) {
            stage = 0;
            phase ^= 1;
          }
        }
      }
    producer_done:;
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      constexpr uint32_t idesc = tc::idesc_bf16_f32(BM, BN);
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      for (int64_t t = t_begin; t < t_end; ++t) {
        if (!tc::mbar_wait(&tempty[acc], acc_phase ^ 1, abort_flag)) break;
        tc::tc_fence_after();
        const uint32_t d_tmem = tmem_base + (uint32_t)(acc * BN);
        bool ok = true;
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
            tc::mma_bf16(d_tmem, tc::sw128_kmajor_desc(a_addr + k * 32), tc::sw128_kmajor_desc(b_addr + k * 32),
                         idesc, (kb | k) != 0 ? 1u : 0u);
          }
          tc::mma_commit(&empty[stage]);
          if (++stage == C::kStages) {
            stage = 0;
            phase ^= 1;
          }
        }
        if (!ok) break;
        tc::mma_commit(&tfull[acc]);
        acc ^= 1;
        if (acc == 0) acc_phase ^= 1;
      }
    }
  } else if (warp >= 4) {
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
      if (row < n) {
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
      const bool row_ok = row < n;
      const uint32_t taddr = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * BN);
#pragma unroll 1
      for (int ch = 0; ch < BN / 32; ++ch) {
        float v[32];
        __syncwarp();
        tc::tmem_ld32(taddr + ch * 32, v);
        const int col0 = ct * BN + ch * 32;
        const float4* sq4 = reinterpret_cast<const float4*>(sqb + col0);
#pragma unroll
        for (int j4 = 0; j4 < 8; ++j4) {
          const float4 sq = __ldg(sq4 + j4);
          const float sj[4] = {sq.x, sq.y, sq.z, sq.w};
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const float s = fmaf(-2.0f, v[j4 * 4 + u], sj[u]);
            const int col = col0 + j4 * 4 + u;
            if (s < tau && row_ok && col != row) {
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
  if (warp == 2) {
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
                  int32_t* __restrict__ out_idx, float* __restrict__ out_dist) {
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
  // exact squared distances of the best L candidates (direct form, FP32)
  const float* xr = X + row * d;
  for (int e = 0; e < PL; ++e) {
    const int j = e < L ? idx[e] : 0x7fffffff;
    float acc = INFINITY;
    if (j != 0x7fffffff) {
      const float* xc = X + (int64_t)j * d;
      acc = 0.f;
      for (int c = lane; c < d; c += 32) {
        const float t = __ldg(xr + c) - __ldg(xc + c);
        acc = fmaf(t, t, acc);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    }
    __syncwarp();
    if (lane == 0) {
      key[e] = acc;
      idx[e] = j;
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

template <int LCAP>
static int launch_topk(const Plan& p, const CUtensorMap& ta, const CUtensorMap& tb, cudaStream_t stream) {
  using C = Cfg<LCAP>;
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr_set[dev]) {
    UMAPB_CUDA_TRY(cudaFuncSetAttribute(topk_kernel<LCAP>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::kSmem),
                   "knn_brute: set smem attribute");
    attr_set[dev] = true;
  }
  topk_kernel<LCAP><<<(unsigned)p.grid, THREADS, C::kSmem, stream>>>(
      ta, tb, p.sqb, (int)p.n, p.num_kb, p.col_tiles, p.tiles, p.slots, p.L, p.cand_s, p.cand_i, p.status);
  UMAPB_LAUNCH_CHECK("knn_brute: topk kernel launch");
  return UMAPB_OK;
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

  UMAPB_CUDA_TRY(cudaMemsetAsync(p.status, 0, sizeof(int32_t), stream), "knn_brute: status reset");
  UMAPB_CUDA_TRY(cudaMemsetAsync(p.cand_i, 0xFF, (size_t)n * p.slots * p.L * sizeof(int32_t), stream),
                 "knn_brute: candidate reset");
  {
    const int64_t warps = p.cols_pad;
    const unsigned blocks = (unsigned)ceil_div(warps * 32, 256);
    knn::prep_kernel<<<blocks, 256, 0, stream>>>(X, n, (int)d, (int)p.ld, p.xb, p.sqb, p.cols_pad);
    UMAPB_LAUNCH_CHECK("knn_brute: prep kernel launch");
  }
  CUtensorMap ta, tb;
  if ((s = make_tmap_bf16_2d(&ta, p.xb, (uint64_t)n, (uint64_t)p.ld, (uint64_t)p.ld, knn::BM, knn::BK))) return s;
  if ((s = make_tmap_bf16_2d(&tb, p.xb, (uint64_t)n, (uint64_t)p.ld, (uint64_t)p.ld, knn::BN, knn::BK))) return s;
  if (p.lcap == 32)
    s = knn::launch_topk<32>(p, ta, tb, stream);
  else if (p.lcap == 64)
    s = knn::launch_topk<64>(p, ta, tb, stream);
  else
    s = knn::launch_topk<128>(p, ta, tb, stream);
  if (s) return s;
  {
    const int P = knn::next_pow2(p.slots * p.L);
    const int PL = knn::next_pow2(p.L);
    const size_t smem = (size_t)knn::RR_WARPS * 2 * P * sizeof(float);
    if (smem > 48 * 1024) {
      static bool set = false;
      if (!set) {
        UMAPB_CUDA_TRY(cudaFuncSetAttribute(knn::rerank_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)(200 * 1024)),
                       "knn_brute: rerank smem attribute");
        set = true;
      }
    }
    const unsigned blocks = (unsigned)ceil_div(n, knn::RR_WARPS);
    knn::rerank_kernel<<<blocks, knn::RR_WARPS * 32, smem, stream>>>(X, n, (int)d, p.cand_s, p.cand_i, p.slots,
                                                                      p.L, P, PL, k, squared, out_idx, out_dist);
    UMAPB_LAUNCH_CHECK("knn_brute: rerank kernel launch");
  }
  return UMAPB_OK;
}
