// BF16 tensor-core GEMM with fused MLP epilogues, for the learned warm-start
// encoder (no counterpart in the reference; its nearest idiom is the MMAE MLP,
// mlx_vis/_mmae/mmae.py:22-38, 258-281).
//
//   C[M, N] = sum_k A[m, k] B[n, k]      A (M x K), B (N x K): BF16, K-major
//
// One CTA per 128 x 128 output tile and K slice (gridDim.z slices of the K
// blocks; the F32 epilogue then writes each slice's partial tile to its own
// M x ldc block of C, for the consumer to sum): warp 0
// streams 64-wide K blocks of A and B with TMA (128-byte swizzle, zero fill past
// M, N, K) through 4 stages, one thread of warp 1 issues tcgen05.mma (M=128, N=128,
// K=16, FP32 accumulation in TMEM), warps 2-5 (one per TMEM lane quarter) read the
// accumulator with tcgen05.ld, 32 columns at a time, and apply the epilogue:
//   EPI_F32        C (f32, row-major, pitch ldc); with K slices, slice z at C + z M ldc
//   EPI_BIAS_GELU  z = C + bias[n]; Z (f32), H = bf16(gelu(z)) row-major and,
//                  when HT != null, its transpose H^T (N x M, pitch ldt)
//   EPI_GELU_BACK  g = C; dZ = g * gelu'(Z) -> bf16 row-major, optional transpose,
//                  optional column sums of the bf16 values in colsum
// The accumulator rows sit one per thread; each 32 x 32 chunk passes through
// shared memory (the drained operand stages) so row-major outputs are written a
// row per warp instruction, and the transposed output straight from the row
// layout, a column per instruction.
// gelu(z) = z * Phi(z); gelu'(z) = Phi(z) + z phi(z) (gelu.cuh).
// Every mbarrier wait is bounded (2 s) and reports through *status.
#include <cuda_bf16.h>
#include <math.h>

#include "common.cuh"
#include "gelu.cuh"
#include "tc.cuh"

namespace umapb {
namespace gemm {

constexpr int BM = 128, BN = 128, BK = 64, UK = 16, STAGES = 4;
constexpr int A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int THREADS = 192;  // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue (lane quarters 2, 3, 0, 1)
constexpr int SMEM = 1024 + STAGES * STAGE_BYTES + 256;

enum Epi : int { EPI_F32 = 0, EPI_BIAS_GELU = 1, EPI_GELU_BACK = 2 };

struct EpiArgs {
  int M, N;
  float* C;  // EPI_F32 output
  int ldc;
  const float* bias;      // EPI_BIAS_GELU
  float* Z;               // EPI_BIAS_GELU output / EPI_GELU_BACK input (pre-activation), pitch ldz
  int ldz;
  __nv_bfloat16* H;       // bf16 output (row-major, pitch ldh)
  int ldh;
  __nv_bfloat16* HT;      // optional bf16 transposed output (N x M, pitch ldt)
  int ldt;
  float* colsum;          // EPI_GELU_BACK: optional column sums of H (atomic adds)
  int64_t slice;          // EPI_F32 with K slices: slice z is written at C + z * slice
};


template <int EPI>
__global__ void __launch_bounds__(THREADS, 1)
    gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int num_kb,
                EpiArgs e, int32_t* __restrict__ status) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* full = bars;
  uint64_t* empty = bars + STAGES;
  uint64_t* done = bars + 2 * STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  // this CTA's K blocks [kb0, kb1); the host sizes the slices so none is empty
  const int per = (num_kb + gridDim.z - 1) / gridDim.z;
  const int kb0 = blockIdx.z * per;
  const int kb1 = kb0 + per < num_kb ? kb0 + per : num_kb;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(done, 1);
    *abort_flag = 0;
    tc::fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    tc::prefetch_tmap(&tmA);
    tc::prefetch_tmap(&tmB);
  }
  if (warp == 2) tc::tmem_alloc(tmem_slot, BN);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      for (int kb = kb0; kb < kb1; ++kb) {
        const int i = kb - kb0;
        const int s = i % STAGES;
        const uint32_t ph = (uint32_t)(i / STAGES) & 1u;
        if (!tc::mbar_wait(&empty[s], ph ^ 1u, abort_flag)) break;
        uint8_t* sa = smem + s * STAGE_BYTES;
        tc::mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
        tc::tma_load_2d(sa, &tmA, &full[s], kb * BK, m0);
        tc::tma_load_2d(sa + A_BYTES, &tmB, &full[s], kb * BK, n0);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = tc::idesc_bf16_f32(BM, BN);
      bool ok = true;
      for (int kb = kb0; kb < kb1; ++kb) {
        const int i = kb - kb0;
        const int s = i % STAGES;
        const uint32_t ph = (uint32_t)(i / STAGES) & 1u;
        if (!tc::mbar_wait(&full[s], ph, abort_flag)) {
          ok = false;
          break;
        }
        tc::tc_fence_after();
        const uint32_t a_addr = tc::smem_u32(smem + s * STAGE_BYTES);
        const uint32_t b_addr = a_addr + A_BYTES;
#pragma unroll
        for (int k = 0; k < BK / UK; ++k)
          tc::mma_bf16(tmem_base, tc::sw128_kmajor_desc(a_addr + k * 32), tc::sw128_kmajor_desc(b_addr + k * 32),
                       idesc, (i | k) != 0 ? 1u : 0u);
        tc::mma_commit(&empty[s]);
      }
      if (ok) tc::mma_commit(done);
    }
  } else {
    // epilogue: thread = accumulator row (TMEM lane), 32 columns per tcgen05.ld,
    // staged through this warp's 32 x 33 float tile in the drained stage memory
    // (every MMA, and so every TMA load, has completed once `done` fires)
    const int q = warp & 3;
    const int rbase = m0 + q * 32;  // first row of this warp's quarter
    float* S = reinterpret_cast<float*>(smem) + q * 32 * 33;
    if (tc::mbar_wait(done, 0, abort_flag)) {
      tc::tc_fence_after();
      for (int ch = 0; ch < BN / 32; ++ch) {
        float v[32];
        __syncwarp();
        tc::tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(ch * 32), v);
        const int nb = n0 + ch * 32;
#pragma unroll
        for (int j = 0; j < 32; ++j) S[lane * 33 + j] = v[j];
        __syncwarp();
        // column phase: lane = column n, one accumulator row per step
        const int n = nb + lane;
        const bool nin = n < e.N;
        float bias_n = 0.f, csum = 0.f;
        if (EPI == EPI_BIAS_GELU && nin) bias_n = e.bias[n];
        float zpre[32];  // GELU_BACK: this column's 32 pre-activations, all loads issued first
        if (EPI == EPI_GELU_BACK) {
#pragma unroll
          for (int rr = 0; rr < 32; ++rr)
            zpre[rr] = (nin && rbase + rr < e.M) ? e.Z[(int64_t)(rbase + rr) * e.ldz + n] : 0.f;
        }
        for (int rr = 0; rr < 32; ++rr) {
          const int m = rbase + rr;
          if (m >= e.M || !nin) continue;
          const float val = S[rr * 33 + lane];
          if (EPI == EPI_F32) {
            e.C[blockIdx.z * e.slice + (int64_t)m * e.ldc + n] = val;
          } else if (EPI == EPI_BIAS_GELU) {
            const float z = val + bias_n;
            e.Z[(int64_t)m * e.ldz + n] = z;
            const __nv_bfloat16 h = __float2bfloat16_rn(gelu(z));
            e.H[(int64_t)m * e.ldh + n] = h;
            S[rr * 33 + lane] = __bfloat162float(h);
          } else {
            const __nv_bfloat16 h = __float2bfloat16_rn(val * gelu_grad(zpre[rr]));
            e.H[(int64_t)m * e.ldh + n] = h;
            const float hf = __bfloat162float(h);
            S[rr * 33 + lane] = hf;
            csum += hf;
          }
        }
        if (EPI == EPI_GELU_BACK && e.colsum && nin) atomicAdd(&e.colsum[n], csum);
        if (EPI != EPI_F32 && e.HT) {  // row phase: lane = row m, one column per step
          __syncwarp();
          const int m = rbase + lane;
          if (m < e.M) {
            for (int j = 0; j < 32 && nb + j < e.N; ++j)
              e.HT[(int64_t)(nb + j) * e.ldt + m] = __float2bfloat16_rn(S[lane * 33 + j]);
          }
        }
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem_base, BN);
  }
  if (threadIdx.x == 0 && *abort_flag) atomicExch(status, (int32_t)kDevTimeoutEpilogue);
}

// Split-precision products: A and B hold three BF16 parts per value,
// x = x0 + x1 + x2 (x0 = bf16(x), x1 = bf16(x - x0), x2 = bf16(x - x0 - x1)), side
// by side at column offsets 0, kp and 2 kp of each row.  A stage holds all six part
// tiles of one 64-wide K block (A0 A1 A2 B0 B1 B2, 96 KB; two stages), loaded once,
// and the MMA thread issues the pairs (0,0) (0,1) (1,0) (0,2) (2,0) (1,1) from them
// into one FP32 TMEM tile: the dropped terms are below 2^-24 of |a||b|, so C carries
// FP32-level error.  K slices (gridDim.z) cut the K blocks; the F32 epilogue writes
// slice z at C + z * slice.
constexpr int S3_TILE = BM * BK * 2;              // one 128 x 64 BF16 part tile (BM == BN)
constexpr int S3_STAGES = 2;
constexpr int S3_STAGE_BYTES = 6 * S3_TILE;
constexpr int S3_SMEM = 1024 + S3_STAGES * S3_STAGE_BYTES + 256;
static_assert(BM == BN, "the split kernel's part tiles share one size");

__global__ void __launch_bounds__(THREADS, 1)
    split3_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int num_kb,
                  EpiArgs e, int32_t* __restrict__ status, int kp) {
  constexpr int kPa[6] = {0, 0, 1, 0, 2, 1};
  constexpr int kPb[6] = {0, 1, 0, 2, 0, 1};
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S3_STAGES * S3_STAGE_BYTES);
  uint64_t* full = bars;
  uint64_t* empty = bars + S3_STAGES;
  uint64_t* done = bars + 2 * S3_STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // blockIdx.x walks the N tiles, so CTAs launched together share an A tile in L2
  const int n0 = blockIdx.x * BN, m0 = blockIdx.y * BM;
  const int per = (num_kb + gridDim.z - 1) / gridDim.z;  // the host sizes the slices so none is empty
  const int kb0 = blockIdx.z * per;
  const int kb1 = kb0 + per < num_kb ? kb0 + per : num_kb;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S3_STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(done, 1);
    *abort_flag = 0;
    tc::fence_mbar_init();
  }
  if (warp == 0 && lane == 0) {
    tc::prefetch_tmap(&tmA);
    tc::prefetch_tmap(&tmB);
  }
  if (warp == 2) tc::tmem_alloc(tmem_slot, BN);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      for (int kb = kb0; kb < kb1; ++kb) {
        const int i = kb - kb0;
        const int s = i % S3_STAGES;
        const uint32_t ph = (uint32_t)(i / S3_STAGES) & 1u;
        if (!tc::mbar_wait(&empty[s], ph ^ 1u, abort_flag)) break;
        uint8_t* st = smem + s * S3_STAGE_BYTES;
        tc::mbar_arrive_expect_tx(&full[s], S3_STAGE_BYTES);
#pragma unroll
        for (int p = 0; p < 3; ++p) {
          tc::tma_load_2d(st + p * S3_TILE, &tmA, &full[s], p * kp + kb * BK, m0);
          tc::tma_load_2d(st + (3 + p) * S3_TILE, &tmB, &full[s], p * kp + kb * BK, n0);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = tc::idesc_bf16_f32(BM, BN);
      bool ok = true;
      for (int kb = kb0; kb < kb1; ++kb) {
        const int i = kb - kb0;
        const int s = i % S3_STAGES;
        const uint32_t ph = (uint32_t)(i / S3_STAGES) & 1u;
        if (!tc::mbar_wait(&full[s], ph, abort_flag)) {
          ok = false;
          break;
        }
        tc::tc_fence_after();
        const uint32_t st = tc::smem_u32(smem + s * S3_STAGE_BYTES);
#pragma unroll
        for (int pr = 0; pr < 6; ++pr) {
          const uint32_t a_addr = st + kPa[pr] * S3_TILE, b_addr = st + (3 + kPb[pr]) * S3_TILE;
#pragma unroll
          for (int k = 0; k < BK / UK; ++k)
            tc::mma_bf16(tmem_base, tc::sw128_kmajor_desc(a_addr + k * 32), tc::sw128_kmajor_desc(b_addr + k * 32),
                         idesc, (i | pr | k) != 0 ? 1u : 0u);
        }
        tc::mma_commit(&empty[s]);
      }
      if (ok) tc::mma_commit(done);
    }
  } else {
    // epilogue: thread = accumulator row (TMEM lane), 32 columns per tcgen05.ld,
    // staged through this warp's 32 x 33 float tile in the drained stage memory so a
    // warp instruction writes 32 consecutive columns of one row
    const int q = warp & 3;
    const int rbase = m0 + q * 32;
    float* S = reinterpret_cast<float*>(smem) + q * 32 * 33;
    if (tc::mbar_wait(done, 0, abort_flag)) {
      tc::tc_fence_after();
      float* C = e.C + blockIdx.z * e.slice;
      for (int ch = 0; ch < BN / 32 && n0 + ch * 32 < e.N; ++ch) {
        float v[32];
        __syncwarp();
        tc::tmem_ld32(tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(ch * 32), v);
#pragma unroll
        for (int j = 0; j < 32; ++j) S[lane * 33 + j] = v[j];
        __syncwarp();
        const int n = n0 + ch * 32 + lane;
        if (n < e.N)
          for (int rr = 0; rr < 32 && rbase + rr < e.M; ++rr) C[(int64_t)(rbase + rr) * e.ldc + n] = S[rr * 33 + lane];
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc::tc_fence_after();
    tc::tmem_dealloc(tmem_base, BN);
  }
  if (threadIdx.x == 0 && *abort_flag) atomicExch(status, (int32_t)kDevTimeoutEpilogue);
}

template <int EPI>
static int launch(const void* A, const void* B, int M, int N, int K, int lda, int ldb, int ksplit, const EpiArgs& e,
                  int32_t* status, cudaStream_t stream) {
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr[dev]) {
    UMAPB_CUDA_TRY(cudaFuncSetAttribute(gemm_kernel<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM),
                   "gemm: smem attribute");
    attr[dev] = true;
  }
  CUtensorMap ta, tb;
  int s;
  if ((s = make_tmap_bf16_2d(&ta, A, (uint64_t)M, (uint64_t)K, (uint64_t)lda, BM, BK))) return s;
  if ((s = make_tmap_bf16_2d(&tb, B, (uint64_t)N, (uint64_t)K, (uint64_t)ldb, BN, BK))) return s;
  const int num_kb = (int)ceil_div(K, BK);
  const int per = (int)ceil_div(num_kb, ksplit);
  const int slices = (int)ceil_div(num_kb, per);  // every slice gets at least one K block
  if (slices < ksplit)  // the caller sums ksplit slices: the ones without K blocks hold zeros
    UMAPB_CUDA_TRY(cudaMemsetAsync(e.C + slices * e.slice, 0, sizeof(float) * (size_t)(ksplit - slices) * e.slice,
                                   stream),
                   "gemm: empty slices");
  dim3 grid((unsigned)ceil_div(M, BM), (unsigned)ceil_div(N, BN), (unsigned)slices);
  gemm_kernel<EPI><<<grid, THREADS, SMEM, stream>>>(ta, tb, num_kb, e, status);
  UMAPB_LAUNCH_CHECK("gemm kernel launch");
  count_launches(1);
  return UMAPB_OK;
}

}  // namespace gemm
}  // namespace umapb

using namespace umapb;

extern "C" int umapb_gemm_bf16(const void* A, const void* B, int32_t M, int32_t N, int32_t K, int32_t lda,
                               int32_t ldb, int32_t epilogue, int32_t ksplit, float* C, int32_t ldc, const float* bias,
                               float* Z, int32_t ldz, void* H, int32_t ldh, void* HT, int32_t ldt, float* colsum,
                               int32_t* status, umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(A && B && status, "gemm: null operand");
  UMAPB_REQUIRE(M >= 1 && N >= 1 && K >= 1, "gemm: empty shape");
  UMAPB_REQUIRE(lda >= K && ldb >= K && lda % 8 == 0 && ldb % 8 == 0,
                "gemm: lda/ldb must be >= K and multiples of 8 elements (16-byte rows)");
  UMAPB_REQUIRE(ksplit >= 1 && ksplit <= 64, "gemm: ksplit must be in [1, 64]");
  UMAPB_REQUIRE(ksplit == 1 || epilogue == gemm::EPI_F32, "gemm: K slices need the F32 epilogue");
  gemm::EpiArgs e{M, N, C, ldc, bias, Z, ldz, static_cast<__nv_bfloat16*>(H), ldh, static_cast<__nv_bfloat16*>(HT),
                  ldt, colsum, (int64_t)M * ldc};
  switch (epilogue) {
    case gemm::EPI_F32:
      UMAPB_REQUIRE(C && ldc >= N, "gemm: EPI_F32 needs C with ldc >= N");
      return gemm::launch<gemm::EPI_F32>(A, B, M, N, K, lda, ldb, ksplit, e, status, stream);
    case gemm::EPI_BIAS_GELU:
      UMAPB_REQUIRE(bias && Z && H && ldz >= N && ldh >= N && (!HT || ldt >= M),
                    "gemm: EPI_BIAS_GELU needs bias, Z and H (and ldt >= M for HT)");
      return gemm::launch<gemm::EPI_BIAS_GELU>(A, B, M, N, K, lda, ldb, 1, e, status, stream);
    case gemm::EPI_GELU_BACK:
      UMAPB_REQUIRE(Z && H && ldz >= N && ldh >= N && (!HT || ldt >= M),
                    "gemm: EPI_GELU_BACK needs Z and H (and ldt >= M for HT)");
      if (colsum) UMAPB_CUDA_TRY(cudaMemsetAsync(colsum, 0, sizeof(float) * N, stream), "gemm: colsum reset");
      return gemm::launch<gemm::EPI_GELU_BACK>(A, B, M, N, K, lda, ldb, 1, e, status, stream);
    default:
      return set_error(UMAPB_ERR_ARG, "gemm: unknown epilogue %d", epilogue);
  }
}

extern "C" int umapb_gemm_split3(const void* A3, const void* B3, int32_t M, int32_t N, int32_t kp, int32_t ksplit,
                                 float* C, int32_t ldc, int32_t* status, umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(A3 && B3 && C && status, "gemm_split3: null argument");
  UMAPB_REQUIRE(M >= 1 && N >= 1 && kp >= gemm::BK && kp % gemm::BK == 0,
                "gemm_split3: need M, N >= 1 and kp a positive multiple of 64");
  UMAPB_REQUIRE((int64_t)kp * 3 < ((int64_t)1 << 31), "gemm_split3: kp too large");
  UMAPB_REQUIRE(ldc >= N, "gemm_split3: ldc must be >= N");
  UMAPB_REQUIRE(ksplit >= 1 && ksplit <= 4096, "gemm_split3: ksplit must be in [1, 4096]");
  static bool attr[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !attr[dev]) {
    UMAPB_CUDA_TRY(cudaFuncSetAttribute(gemm::split3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        gemm::S3_SMEM),
                   "gemm_split3: smem attribute");
    attr[dev] = true;
  }
  CUtensorMap ta, tb;
  int s;
  const uint64_t w = (uint64_t)kp * 3;
  if ((s = make_tmap_bf16_2d(&ta, A3, (uint64_t)M, w, w, gemm::BM, gemm::BK))) return s;
  if ((s = make_tmap_bf16_2d(&tb, B3, (uint64_t)N, w, w, gemm::BN, gemm::BK))) return s;
  const int num_kb = kp / gemm::BK;
  const int per = (int)ceil_div(num_kb, ksplit);
  const int slices = (int)ceil_div(num_kb, per);  // every slice gets at least one K block
  gemm::EpiArgs e{M, N, C, ldc, nullptr, nullptr, 0, nullptr, 0, nullptr, 0, nullptr, (int64_t)M * ldc};
  if (slices < ksplit)  // the caller sums ksplit slices: the ones without K blocks hold zeros
    UMAPB_CUDA_TRY(cudaMemsetAsync(C + slices * e.slice, 0, sizeof(float) * (size_t)(ksplit - slices) * e.slice,
                                   stream),
                   "gemm_split3: empty slices");
  dim3 grid((unsigned)ceil_div(N, gemm::BN), (unsigned)ceil_div(M, gemm::BM), (unsigned)slices);
  gemm::split3_kernel<<<grid, gemm::THREADS, gemm::S3_SMEM, stream>>>(ta, tb, num_kb, e, status, kp);
  UMAPB_LAUNCH_CHECK("gemm_split3 kernel launch");
  count_launches(1);
  return UMAPB_OK;
}
