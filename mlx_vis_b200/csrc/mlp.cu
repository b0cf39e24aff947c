// Learned warm-start encoder d -> 512 -> 512 -> c (GELU), the pieces around the
// tensor-core GEMMs of gemm.cu.  New work: the reference has no learned layout
// initialisation; its closest idiom is the MMAE MLP and AdamW step
// (mlx_vis/_mmae/mmae.py:22-38, 258-281).
//
// Training step (batch B, MSE between the encoder output Y and the target T):
//   X (f32)  --convert-->  Xb (bf16, B x ldx) and X^T (bf16, d x B)
//   Z1 = Xb W1^T + b1, H1 = gelu(Z1)          gemm EPI_BIAS_GELU  (+ H1^T)
//   Z2 = H1 W2^T + b2, H2 = gelu(Z2)          gemm EPI_BIAS_GELU  (+ H2^T)
//   Y  = H2 W3^T + b3                         head_forward (c <= 4, FP32 weights)
//   loss = mean_b |Y - T|^2, dY = 2 (Y - T) / B
//   dW3 = dY^T H2, db3 = sum dY, dZ2 = (dY W3) * gelu'(Z2)   head_backward
//   dW2 = dZ2^T H1 (gemm, K = B), db2 = column sums of dZ2
//   dZ1 = (dZ2 W2) * gelu'(Z1)                gemm EPI_GELU_BACK with W2^T
//   dW1 = dZ1^T X (gemm, K = B), db1 = column sums of dZ1
//   AdamW on the FP32 master weights, then BF16 copies (and W2^T) for the GEMMs.
#include <cuda_bf16.h>
#include <math.h>

#include "common.cuh"

namespace umapb {
namespace mlp {

constexpr int kMaxOut = 4;

// X (rows x d, f32) -> Xb (rows x ldx bf16, zero padded) and optional XT (d x rows bf16, pitch ldt)
__global__ void convert_kernel(const float* __restrict__ X, int rows, int d, int ldx, __nv_bfloat16* __restrict__ Xb,
                               __nv_bfloat16* __restrict__ XT, int ldt) {
  __shared__ float tile[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int i = ty; i < 32; i += 8) {
    const int r = r0 + i, c = c0 + tx;
    float v = 0.f;
    if (r < rows && c < d) v = X[(int64_t)r * d + c];
    if (r < rows && c < ldx) Xb[(int64_t)r * ldx + c] = __float2bfloat16_rn(v);
    tile[i][tx] = v;
  }
  if (!XT) return;
  __syncthreads();
  for (int i = ty; i < 32; i += 8) {
    const int c = c0 + i, r = r0 + tx;
    if (c < d && r < rows) XT[(int64_t)c * ldt + r] = __float2bfloat16_rn(tile[tx][i]);
  }
}

// Y[b] = H[b] . W^T + bias, one warp per row
__global__ void head_forward_kernel(const __nv_bfloat16* __restrict__ H, int ldh, int B, int Hd,
                                    const float* __restrict__ W, const float* __restrict__ bias, int c,
                                    float* __restrict__ Y) {
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (row >= B) return;
  float acc[kMaxOut] = {0.f, 0.f, 0.f, 0.f};
  for (int i = lane; i < Hd; i += 32) {
    const float h = __bfloat162float(H[(int64_t)row * ldh + i]);
    for (int o = 0; o < c; ++o) acc[o] = fmaf(h, W[o * Hd + i], acc[o]);
  }
  for (int o = 0; o < c; ++o) {
    float s = acc[o];
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) s += __shfl_xor_sync(0xffffffffu, s, sh);
    if (lane == 0) Y[(int64_t)row * c + o] = s + bias[o];
  }
}

// dY = 2 (Y - T) / B; loss += sum (Y - T)^2 / B; dZ2 = (dY W3) * gelu'(Z2) (bf16 + transpose)
__global__ void head_backward_rows_kernel(const float* __restrict__ Y, const float* __restrict__ T, int B, int c,
                                          const float* __restrict__ W, int Hd, const float* __restrict__ Z, int ldz,
                                          float* __restrict__ dY, __nv_bfloat16* __restrict__ dZ, int lddz,
                                          __nv_bfloat16* __restrict__ dZT, int ldt, float* __restrict__ loss) {
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (row >= B) return;
  float g[kMaxOut];
  float l = 0.f;
  for (int o = 0; o < c; ++o) {
    const float diff = Y[(int64_t)row * c + o] - T[(int64_t)row * c + o];
    g[o] = 2.0f * diff / (float)B;
    l += diff * diff;
  }
  if (lane < c) dY[(int64_t)row * c + lane] = g[lane < c ? lane : 0];
  if (lane == 0) atomicAdd(loss, l / (float)B);
  for (int i = lane; i < Hd; i += 32) {
    float s = 0.f;
    for (int o = 0; o < c; ++o) s = fmaf(g[o], W[o * Hd + i], s);
    const float z = Z[(int64_t)row * ldz + i];
    const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
    const __nv_bfloat16 v = __float2bfloat16_rn(s * (cdf + z * pdf));
    dZ[(int64_t)row * lddz + i] = v;
    dZT[(int64_t)i * ldt + row] = v;
  }
}

// out[n] = sum over the row n of M^T (N x B, pitch ld) — one warp per n
__global__ void rowsum_bf16_kernel(const __nv_bfloat16* __restrict__ MT, int N, int B, int ld, float* __restrict__ out) {
  const int n = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (n >= N) return;
  float s = 0.f;
  for (int b = lane; b < B; b += 32) s += __bfloat162float(MT[(int64_t)n * ld + b]);
#pragma unroll
  for (int sh = 16; sh > 0; sh >>= 1) s += __shfl_xor_sync(0xffffffffu, s, sh);
  if (lane == 0) out[n] = s;
}

// dW3[o][i] = sum_b dY[b][o] H2T[i][b]; db3[o] = sum_b dY[b][o].  One warp per i.
__global__ void head_weight_grad_kernel(const float* __restrict__ dY, int B, int c, const __nv_bfloat16* __restrict__ HT,
                                        int ld, int Hd, float* __restrict__ dW, float* __restrict__ db) {
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (i > Hd) return;
  float acc[kMaxOut] = {0.f, 0.f, 0.f, 0.f};
  for (int b = lane; b < B; b += 32) {
    const float h = i < Hd ? __bfloat162float(HT[(int64_t)i * ld + b]) : 1.0f;  // row Hd: bias
    for (int o = 0; o < c; ++o) acc[o] = fmaf(dY[(int64_t)b * c + o], h, acc[o]);
  }
  for (int o = 0; o < c; ++o) {
    float s = acc[o];
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) s += __shfl_xor_sync(0xffffffffu, s, sh);
    if (lane == 0) {
      if (i < Hd) dW[o * Hd + i] = s;
      else db[o] = s;
    }
  }
}

// Decoupled-weight-decay Adam (AdamW) on FP32 masters; optional BF16 copy (rows x cols,
// pitch ldb) and transposed BF16 copy (cols x rows, pitch ldbt).
__global__ void adamw_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                             float* __restrict__ v, int64_t count, float lr, float beta1, float beta2, float eps,
                             float wd, float bc1, float bc2, int cols, __nv_bfloat16* __restrict__ pb, int ldb,
                             __nv_bfloat16* __restrict__ pbt, int ldbt, int rows) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += (int64_t)gridDim.x * blockDim.x) {
    const float gr = g[t];
    const float mt = beta1 * m[t] + (1.0f - beta1) * gr;
    const float vt = beta2 * v[t] + (1.0f - beta2) * gr * gr;
    m[t] = mt;
    v[t] = vt;
    float w = p[t] * (1.0f - lr * wd);
    w -= lr * (mt / bc1) / (sqrtf(vt / bc2) + eps);
    p[t] = w;
    const int r = (int)(t / cols), c = (int)(t % cols);
    if (pb) pb[(int64_t)r * ldb + c] = __float2bfloat16_rn(w);
    if (pbt) pbt[(int64_t)c * ldbt + r] = __float2bfloat16_rn(w);
  }
}

}  // namespace mlp
}  // namespace umapb

using namespace umapb;

static unsigned grid_for(int64_t work, int per_block) {
  const int64_t b = ceil_div(work, per_block);
  const int64_t cap = (int64_t)num_sms() * 16;
  return (unsigned)(b < cap ? b : cap);
}

extern "C" int umapb_mlp_convert(const float* X, int32_t rows, int32_t d, int32_t ldx, void* Xb, void* XT,
                                 int32_t ldt, umapb_stream_t stream) {
  clear_error();
  UMAPB_REQUIRE(X && Xb && rows >= 1 && d >= 1 && ldx >= d, "mlp_convert: bad arguments");
  UMAPB_REQUIRE(!XT || ldt >= rows, "mlp_convert: ldt must be >= rows");
  dim3 grid((unsigned)ceil_div(ldx, 32), (unsigned)ceil_div(rows, 32)), block(32, 8);
  mlp::convert_kernel<<<grid, block, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      X, rows, d, ldx, static_cast<__nv_bfloat16*>(Xb), static_cast<__nv_bfloat16*>(XT), ldt);
  UMAPB_LAUNCH_CHECK("mlp_convert kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_mlp_head_forward(const void* H, int32_t ldh, int32_t B, int32_t Hd, const float* W,
                                      const float* bias, int32_t c, float* Y, umapb_stream_t stream) {
  clear_error();
  UMAPB_REQUIRE(H && W && bias && Y && B >= 1 && Hd >= 1 && ldh >= Hd, "mlp_head_forward: bad arguments");
  UMAPB_REQUIRE(c >= 1 && c <= mlp::kMaxOut, "mlp_head_forward: 1 <= c <= 4");
  mlp::head_forward_kernel<<<(unsigned)ceil_div((int64_t)B * 32, 256), 256, 0,
                             reinterpret_cast<cudaStream_t>(stream)>>>(static_cast<const __nv_bfloat16*>(H), ldh, B,
                                                                       Hd, W, bias, c, Y);
  UMAPB_LAUNCH_CHECK("mlp_head_forward kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_mlp_head_backward(const float* Y, const float* T, int32_t B, int32_t c, const float* W, int32_t Hd,
                                       const float* Z2, int32_t ldz, const void* H2T, int32_t ldt, float* dY,
                                       float* dW, float* db, void* dZ2, int32_t lddz, void* dZ2T, float* loss,
                                       umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(Y && T && W && Z2 && H2T && dY && dW && db && dZ2 && dZ2T && loss, "mlp_head_backward: null argument");
  UMAPB_REQUIRE(c >= 1 && c <= mlp::kMaxOut && B >= 1 && Hd >= 1 && ldz >= Hd && lddz >= Hd && ldt >= B,
                "mlp_head_backward: bad shape");
  UMAPB_CUDA_TRY(cudaMemsetAsync(loss, 0, sizeof(float), stream), "mlp_head_backward: loss reset");
  mlp::head_backward_rows_kernel<<<(unsigned)ceil_div((int64_t)B * 32, 256), 256, 0, stream>>>(
      Y, T, B, c, W, Hd, Z2, ldz, dY, static_cast<__nv_bfloat16*>(dZ2), lddz, static_cast<__nv_bfloat16*>(dZ2T), ldt,
      loss);
  mlp::head_weight_grad_kernel<<<(unsigned)ceil_div((int64_t)(Hd + 1) * 32, 256), 256, 0, stream>>>(
      dY, B, c, static_cast<const __nv_bfloat16*>(H2T), ldt, Hd, dW, db);
  UMAPB_LAUNCH_CHECK("mlp_head_backward kernels");
  count_launches(2);
  return UMAPB_OK;
}

extern "C" int umapb_mlp_rowsum(const void* MT, int32_t N, int32_t B, int32_t ld, float* out, umapb_stream_t stream) {
  clear_error();
  UMAPB_REQUIRE(MT && out && N >= 1 && B >= 1 && ld >= B, "mlp_rowsum: bad arguments");
  mlp::rowsum_bf16_kernel<<<(unsigned)ceil_div((int64_t)N * 32, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      static_cast<const __nv_bfloat16*>(MT), N, B, ld, out);
  UMAPB_LAUNCH_CHECK("mlp_rowsum kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_adamw(float* p, const float* g, float* m, float* v, int32_t rows, int32_t cols, float lr,
                           float beta1, float beta2, float eps, float weight_decay, int32_t step, void* p_bf16,
                           int32_t ldb, void* p_bf16_t, int32_t ldbt, umapb_stream_t stream) {
  clear_error();
  UMAPB_REQUIRE(p && g && m && v && rows >= 1 && cols >= 1 && step >= 1, "adamw: bad arguments");
  UMAPB_REQUIRE(!p_bf16 || ldb >= cols, "adamw: ldb must be >= cols");
  UMAPB_REQUIRE(!p_bf16_t || ldbt >= rows, "adamw: ldbt must be >= rows");
  const float bc1 = 1.0f - powf(beta1, (float)step), bc2 = 1.0f - powf(beta2, (float)step);
  const int64_t count = (int64_t)rows * cols;
  mlp::adamw_kernel<<<grid_for(count, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      p, g, m, v, count, lr, beta1, beta2, eps, weight_decay, bc1, bc2, cols, static_cast<__nv_bfloat16*>(p_bf16), ldb,
      static_cast<__nv_bfloat16*>(p_bf16_t), ldbt, rows);
  UMAPB_LAUNCH_CHECK("adamw kernel");
  count_launches(1);
  return UMAPB_OK;
}
