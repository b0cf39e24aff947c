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
//   dW3 = dY^T H2, db3 = sum dY, dZ2 = (dY W3) * gelu'(Z2) (+ dZ2^T),
//   db2 = column sums of dZ2                                head_backward
//   dW2 = dZ2^T H1 (gemm, K = B, K slices)
//   dZ1 = (dZ2 W2) * gelu'(Z1) (+ dZ1^T, db1)  gemm EPI_GELU_BACK with W2^T
//   dW1 = dZ1^T X (gemm, K = B, K slices)
//   AdamW on all FP32 master weights in one launch, with their BF16 copies (and
//   W2^T) for the GEMMs.
#include <cuda_bf16.h>
#include <math.h>

#include "common.cuh"
#include "gelu.cuh"

namespace umapb {
namespace mlp {

constexpr int kMaxOut = 4;

// X (rows x d, f32) -> Xb (rows x ldx bf16, zero padded) and optional XT (d x rows bf16, pitch ldt)
// (row r of the outputs reads row row_idx[r] of X when row_idx is given)
__global__ void convert_kernel(const float* __restrict__ X, const int64_t* __restrict__ row_idx, int rows, int d,
                               int ldx, __nv_bfloat16* __restrict__ Xb, __nv_bfloat16* __restrict__ XT, int ldt) {
  __shared__ float tile[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int i = ty; i < 32; i += 8) {
    const int r = r0 + i, c = c0 + tx;
    float v = 0.f;
    if (r < rows && c < d) v = X[(row_idx ? row_idx[r] : (int64_t)r) * d + c];
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

// Y[b] = H[b] . W^T + bias, one warp per row; W (c x Hd) staged in shared memory;
// 16-byte loads of H when the rows allow it
__global__ void head_forward_kernel(const __nv_bfloat16* __restrict__ H, int ldh, int B, int Hd,
                                    const float* __restrict__ W, const float* __restrict__ bias, int c,
                                    float* __restrict__ Y) {
  extern __shared__ float Ws[];  // c x Hd
  for (int i = threadIdx.x; i < c * Hd; i += blockDim.x) Ws[i] = W[i];
  __syncthreads();
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (row >= B) return;
  float acc[kMaxOut] = {0.f, 0.f, 0.f, 0.f};
  const __nv_bfloat16* h = H + (int64_t)row * ldh;
  if ((Hd & 7) == 0 && (ldh & 7) == 0 && (reinterpret_cast<uintptr_t>(H) & 15) == 0) {
    for (int q = lane; q < Hd / 8; q += 32) {
      const uint4 u = reinterpret_cast<const uint4*>(h)[q];
      const __nv_bfloat162* p2 = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float2 f = __bfloat1622float2(p2[e]);
        const int i = 8 * q + 2 * e;
        for (int o = 0; o < c; ++o) acc[o] = fmaf(f.y, Ws[o * Hd + i + 1], fmaf(f.x, Ws[o * Hd + i], acc[o]));
      }
    }
  } else {
    for (int i = lane; i < Hd; i += 32) {
      const float f = __bfloat162float(h[i]);
      for (int o = 0; o < c; ++o) acc[o] = fmaf(f, Ws[o * Hd + i], acc[o]);
    }
  }
  for (int o = 0; o < c; ++o) {
    float s = acc[o];
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) s += __shfl_xor_sync(0xffffffffu, s, sh);
    if (lane == 0) Y[(int64_t)row * c + o] = s + bias[o];
  }
}

// One block per 32 rows x 128 columns (8 warps, 4 rows each; a lane owns 4 adjacent
// columns):
//   g = dY[b] = 2 (Y[b] - T[b]) / B (T row t_idx[b] when given) and the loss
//   (column block 0 only),
//   dZ2 = bf16((g W) * gelu'(Z2)) row-major, and transposed through shared memory,
//   dW += g^T H2, db += sum g (column block 0), dbias2 += column sums of dZ2,
// the sums accumulated with atomics (the host entry zeroes them first).
constexpr int kHbRows = 32, kHbCols = 128;
__global__ void __launch_bounds__(256) head_backward_kernel(
    const float* __restrict__ Y, const float* __restrict__ T, const int64_t* __restrict__ t_idx, int B, int c,
    const float* __restrict__ W, int Hd,
    const float* __restrict__ Z, int ldz, const __nv_bfloat16* __restrict__ H2, int ldh2, float* __restrict__ dY,
    float* __restrict__ dW, float* __restrict__ db, __nv_bfloat16* __restrict__ dZ, int lddz,
    __nv_bfloat16* __restrict__ dZT, int ldt, float* __restrict__ dbias2, float* __restrict__ loss) {
  __shared__ float g[kHbRows][kMaxOut];
  __shared__ float tile[kHbRows][kHbCols + 1];
  __shared__ float red[8][kMaxOut + 1][kHbCols];  // per-warp partial dW (c rows) and dbias2 (row kMaxOut)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r0 = blockIdx.y * kHbRows, c0 = blockIdx.x * kHbCols;
  if (threadIdx.x < kHbRows) {
    const int b = r0 + threadIdx.x;
    float l = 0.f;
    for (int o = 0; o < kMaxOut; ++o) {
      float gv = 0.f;
      if (b < B && o < c) {
        const float diff = Y[(int64_t)b * c + o] - T[(t_idx ? t_idx[b] : (int64_t)b) * c + o];
        gv = 2.0f * diff / (float)B;
        l += diff * diff;
        if (blockIdx.x == 0) dY[(int64_t)b * c + o] = gv;
      }
      g[threadIdx.x][o] = gv;
    }
    if (blockIdx.x == 0) {
#pragma unroll
      for (int sh = 16; sh > 0; sh >>= 1) l += __shfl_xor_sync(0xffffffffu, l, sh);
      if (threadIdx.x == 0) atomicAdd(loss, l / (float)B);
      for (int o = 0; o < c; ++o) {
        float gs = g[threadIdx.x][o];
#pragma unroll
        for (int sh = 16; sh > 0; sh >>= 1) gs += __shfl_xor_sync(0xffffffffu, gs, sh);
        if (threadIdx.x == 0) atomicAdd(&db[o], gs);
      }
    }
  }
  __syncthreads();
  const int col0 = c0 + lane * 4;
  float w[kMaxOut][4];
#pragma unroll
  for (int o = 0; o < kMaxOut; ++o)
#pragma unroll
    for (int u = 0; u < 4; ++u) w[o][u] = (o < c && col0 + u < Hd) ? W[o * Hd + col0 + u] : 0.f;
  const bool vec = col0 + 3 < Hd && (ldz & 3) == 0 && (ldh2 & 3) == 0 && (lddz & 3) == 0 &&
                   ((reinterpret_cast<uintptr_t>(Z) | reinterpret_cast<uintptr_t>(H2) |
                     reinterpret_cast<uintptr_t>(dZ)) & 15) == 0;
  float pw[kMaxOut][4] = {}, pb[4] = {0.f, 0.f, 0.f, 0.f};
  for (int k4 = 0; k4 < kHbRows / 8; ++k4) {
    const int rr = warp * (kHbRows / 8) + k4;
    const int b = r0 + rr;
    float z[4] = {0.f, 0.f, 0.f, 0.f}, h2[4] = {0.f, 0.f, 0.f, 0.f}, dz[4] = {0.f, 0.f, 0.f, 0.f};
    if (b < B) {
      if (vec) {
        const float4 z4 = *reinterpret_cast<const float4*>(Z + (int64_t)b * ldz + col0);
        const uint2 hh = *reinterpret_cast<const uint2*>(H2 + (int64_t)b * ldh2 + col0);
        const float2 ha = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&hh.x));
        const float2 hb = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&hh.y));
        z[0] = z4.x, z[1] = z4.y, z[2] = z4.z, z[3] = z4.w;
        h2[0] = ha.x, h2[1] = ha.y, h2[2] = hb.x, h2[3] = hb.y;
      } else {
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (col0 + u < Hd) {
            z[u] = Z[(int64_t)b * ldz + col0 + u];
            h2[u] = __bfloat162float(H2[(int64_t)b * ldh2 + col0 + u]);
          }
      }
      __nv_bfloat16 hv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        float sacc = 0.f;
#pragma unroll
        for (int o = 0; o < kMaxOut; ++o) sacc = fmaf(g[rr][o], w[o][u], sacc);
        hv[u] = __float2bfloat16_rn(sacc * gelu_grad(z[u]));
        dz[u] = col0 + u < Hd ? __bfloat162float(hv[u]) : 0.f;
#pragma unroll
        for (int o = 0; o < kMaxOut; ++o) pw[o][u] = fmaf(g[rr][o], h2[u], pw[o][u]);
      }
      if (vec) {
        uint2 out;
        *reinterpret_cast<__nv_bfloat162*>(&out.x) = __halves2bfloat162(hv[0], hv[1]);
        *reinterpret_cast<__nv_bfloat162*>(&out.y) = __halves2bfloat162(hv[2], hv[3]);
        *reinterpret_cast<uint2*>(dZ + (int64_t)b * lddz + col0) = out;
      } else {
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (col0 + u < Hd) dZ[(int64_t)b * lddz + col0 + u] = hv[u];
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      pb[u] += dz[u];
      tile[rr][lane * 4 + u] = dz[u];
    }
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
#pragma unroll
    for (int o = 0; o < kMaxOut; ++o) red[warp][o][lane * 4 + u] = pw[o][u];
    red[warp][kMaxOut][lane * 4 + u] = pb[u];
  }
  __syncthreads();
  // column sums over the 8 warps, then one atomic per column and output
  for (int t = threadIdx.x; t < kHbCols; t += blockDim.x) {
    const int col = c0 + t;
    if (col >= Hd) continue;
    float sb = 0.f;
    for (int w8 = 0; w8 < 8; ++w8) sb += red[w8][kMaxOut][t];
    atomicAdd(&dbias2[col], sb);
    for (int o = 0; o < c; ++o) {
      float sw = 0.f;
      for (int w8 = 0; w8 < 8; ++w8) sw += red[w8][o][t];
      atomicAdd(&dW[o * Hd + col], sw);
    }
  }
  // dZ^T: a warp writes one column at a time, lane = row (64 contiguous bytes)
  for (int t = warp; t < kHbCols; t += 8) {
    const int col = c0 + t, b = r0 + lane;
    if (col < Hd && b < B) dZT[(int64_t)col * ldt + b] = __float2bfloat16_rn(tile[lane][t]);
  }
}

// Decoupled-weight-decay Adam (AdamW) on FP32 masters, every parameter group in one
// launch; a group's gradient may arrive as K slices (summed here, the sum kept in
// slice 0); optional BF16 copy (rows x cols, pitch ldb) and transposed BF16 copy
// (cols x rows, pitch ldbt).  The step number t comes from device memory, so a
// captured training step replays with the current count; bias corrections 1 - beta^t.
constexpr int kMaxGroups = 8;
struct AdamwGroups {
  int n;
  int64_t start[kMaxGroups + 1];  // offsets of the groups in the flattened index space
  float* p[kMaxGroups];
  float* g[kMaxGroups];
  int nsplit[kMaxGroups];          // gradient = sum of nsplit slices, stride apart
  int64_t stride[kMaxGroups];
  float* m[kMaxGroups];
  float* v[kMaxGroups];
  int cols[kMaxGroups];
  __nv_bfloat16* pb[kMaxGroups];
  int ldb[kMaxGroups];
  __nv_bfloat16* pbt[kMaxGroups];
  int ldbt[kMaxGroups];
};

__global__ void adamw_kernel(AdamwGroups G, float lr, float beta1, float beta2, float eps, float wd,
                             const int32_t* __restrict__ step) {
  const float tstep = (float)*step;
  const float bc1 = 1.0f - powf(beta1, tstep), bc2 = 1.0f - powf(beta2, tstep);
  const int64_t total = G.start[G.n];
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
    int k = 0;
    while (k + 1 < G.n && t >= G.start[k + 1]) ++k;
    const int i = (int)(t - G.start[k]);  // a group holds < 2^31 values
    float gr = G.g[k][i];
    if (G.nsplit[k] > 1) {  // K-sliced gradient: sum the slices, keep the sum in slice 0
      for (int sl = 1; sl < G.nsplit[k]; ++sl) gr += G.g[k][i + sl * G.stride[k]];
      G.g[k][i] = gr;
    }
    const float mt = beta1 * G.m[k][i] + (1.0f - beta1) * gr;
    const float vt = beta2 * G.v[k][i] + (1.0f - beta2) * gr * gr;
    G.m[k][i] = mt;
    G.v[k][i] = vt;
    float wv = G.p[k][i] * (1.0f - lr * wd);
    wv -= lr * (mt / bc1) / (sqrtf(vt / bc2) + eps);
    G.p[k][i] = wv;
    const int cols = G.cols[k];
    const int r = i / cols, cc = i - r * cols;
    if (G.pb[k]) G.pb[k][(int64_t)r * G.ldb[k] + cc] = __float2bfloat16_rn(wv);
    if (G.pbt[k]) G.pbt[k][(int64_t)cc * G.ldbt[k] + r] = __float2bfloat16_rn(wv);
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

extern "C" int umapb_mlp_convert(const float* X, const int64_t* row_idx, int32_t rows, int32_t d, int32_t ldx,
                                 void* Xb, void* XT, int32_t ldt, umapb_stream_t stream) {
  clear_error();
  UMAPB_REQUIRE(X && Xb && rows >= 1 && d >= 1 && ldx >= d, "mlp_convert: bad arguments");
  UMAPB_REQUIRE(!XT || ldt >= rows, "mlp_convert: ldt must be >= rows");
  dim3 grid((unsigned)ceil_div(ldx, 32), (unsigned)ceil_div(rows, 32)), block(32, 8);
  mlp::convert_kernel<<<grid, block, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      X, row_idx, rows, d, ldx, static_cast<__nv_bfloat16*>(Xb), static_cast<__nv_bfloat16*>(XT), ldt);
  UMAPB_LAUNCH_CHECK("mlp_convert kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_mlp_head_forward(const void* H, int32_t ldh, int32_t B, int32_t Hd, const float* W,
                                      const float* bias, int32_t c, float* Y, umapb_stream_t stream) {
  clear_error();
  UMAPB_REQUIRE(H && W && bias && Y && B >= 1 && Hd >= 1 && ldh >= Hd && c >= 1 && c <= mlp::kMaxOut,
                "mlp_head_forward: bad arguments");
  const size_t smem = sizeof(float) * (size_t)c * Hd;
  UMAPB_REQUIRE(smem <= 48 * 1024, "mlp_head_forward: c * Hd too large");
  mlp::head_forward_kernel<<<(unsigned)ceil_div((int64_t)B * 32, 256), 256, smem,
                             reinterpret_cast<cudaStream_t>(stream)>>>(static_cast<const __nv_bfloat16*>(H), ldh, B,
                                                                       Hd, W, bias, c, Y);
  UMAPB_LAUNCH_CHECK("mlp_head_forward kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_mlp_head_backward(const float* Y, const float* T, const int64_t* t_idx, int32_t B, int32_t c,
                                       const float* W,
                                       int32_t Hd, const float* Z2, int32_t ldz, const void* H2, int32_t ldh2,
                                       float* dY, float* dW, float* db, void* dZ2, int32_t lddz, void* dZ2T,
                                       int32_t ldt, float* dbias2, float* loss, umapb_stream_t stream_) {
  clear_error();
  cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
  UMAPB_REQUIRE(Y && T && W && Z2 && H2 && dY && dW && db && dZ2 && dZ2T && dbias2 && loss,
                "mlp_head_backward: null argument");
  UMAPB_REQUIRE(B >= 1 && c >= 1 && c <= mlp::kMaxOut && Hd >= 1 && ldz >= Hd && ldh2 >= Hd && lddz >= Hd &&
                    ldt >= B,
                "mlp_head_backward: bad shape");
  UMAPB_CUDA_TRY(cudaMemsetAsync(loss, 0, sizeof(float), stream), "mlp_head_backward: loss reset");
  UMAPB_CUDA_TRY(cudaMemsetAsync(dW, 0, sizeof(float) * c * Hd, stream), "mlp_head_backward: dW reset");
  UMAPB_CUDA_TRY(cudaMemsetAsync(db, 0, sizeof(float) * c, stream), "mlp_head_backward: db reset");
  UMAPB_CUDA_TRY(cudaMemsetAsync(dbias2, 0, sizeof(float) * Hd, stream), "mlp_head_backward: dbias2 reset");
  dim3 grid((unsigned)ceil_div(Hd, mlp::kHbCols), (unsigned)ceil_div(B, mlp::kHbRows));
  mlp::head_backward_kernel<<<grid, 256, 0, stream>>>(Y, T, t_idx, B, c, W, Hd, Z2, ldz,
                                                      static_cast<const __nv_bfloat16*>(H2), ldh2, dY, dW, db,
                                                      static_cast<__nv_bfloat16*>(dZ2), lddz,
                                                      static_cast<__nv_bfloat16*>(dZ2T), ldt, dbias2, loss);
  UMAPB_LAUNCH_CHECK("mlp_head_backward kernel");
  count_launches(1);
  return UMAPB_OK;
}

extern "C" int umapb_adamw(int32_t n_groups, float* const* p, float* const* g, const int32_t* g_slices,
                           const int64_t* g_stride, float* const* m, float* const* v, const int32_t* rows,
                           const int32_t* cols, void* const* p_bf16,
                           const int32_t* ldb, void* const* p_bf16_t, const int32_t* ldbt, float lr, float beta1,
                           float beta2, float eps, float weight_decay, const int32_t* step, umapb_stream_t stream) {
  clear_error();
  UMAPB_REQUIRE(n_groups >= 1 && n_groups <= mlp::kMaxGroups, "adamw: need 1 <= n_groups <= 8");
  UMAPB_REQUIRE(p && g && m && v && rows && cols && step, "adamw: null argument");
  mlp::AdamwGroups G{};
  G.n = n_groups;
  G.start[0] = 0;
  for (int k = 0; k < n_groups; ++k) {
    UMAPB_REQUIRE(p[k] && g[k] && m[k] && v[k] && rows[k] >= 1 && cols[k] >= 1, "adamw: bad group");
    UMAPB_REQUIRE((int64_t)rows[k] * cols[k] < ((int64_t)1 << 31), "adamw: group too large");
    void* pb = p_bf16 ? p_bf16[k] : nullptr;
    void* pbt = p_bf16_t ? p_bf16_t[k] : nullptr;
    UMAPB_REQUIRE(!pb || ldb[k] >= cols[k], "adamw: ldb must be >= cols");
    UMAPB_REQUIRE(!pbt || ldbt[k] >= rows[k], "adamw: ldbt must be >= rows");
    G.p[k] = p[k];
    G.g[k] = g[k];
    G.nsplit[k] = g_slices ? g_slices[k] : 1;
    G.stride[k] = g_slices ? g_stride[k] : 0;
    UMAPB_REQUIRE(G.nsplit[k] >= 1 && (G.nsplit[k] == 1 || G.stride[k] >= (int64_t)rows[k] * cols[k]),
                  "adamw: gradient slices need a stride >= rows * cols");
    G.m[k] = m[k];
    G.v[k] = v[k];
    G.cols[k] = cols[k];
    G.pb[k] = static_cast<__nv_bfloat16*>(pb);
    G.ldb[k] = pb ? ldb[k] : 0;
    G.pbt[k] = static_cast<__nv_bfloat16*>(pbt);
    G.ldbt[k] = pbt ? ldbt[k] : 0;
    G.start[k + 1] = G.start[k] + (int64_t)rows[k] * cols[k];
  }
  mlp::adamw_kernel<<<grid_for(G.start[n_groups], 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      G, lr, beta1, beta2, eps, weight_decay, step);
  UMAPB_LAUNCH_CHECK("adamw kernel");
  count_launches(1);
  return UMAPB_OK;
}
