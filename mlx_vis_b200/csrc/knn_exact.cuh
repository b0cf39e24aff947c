// Exact brute-force kNN for long lists (k + extra > 128), the path the fused top-k
// tile kernel does not cover.  Declared here, used by knn_brute.cu's entry points.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace umapb {
namespace knnx {

constexpr int kMaxK = 4096;

struct Plan {
  int64_t n, d, r0, m, R;  // rows, features, query rows [r0, r0 + m), query rows per block
  int k, L, kp;  // L = k + extra candidates, reranked exactly
  size_t bytes;
  int32_t* status;  // first word of the workspace (bounded-wait status of the GEMMs)
  void* x3;         // (n, 3 kp) BF16 split of X
  float* sq;        // (n) squared norms
  float* C;         // (R, n) dot products of one block of query rows
};

// Sizes (ws == nullptr) or carves the workspace; argument errors set the message.
int plan(int64_t n, int64_t d, int k, int L, int64_t r0, int64_t m, void* ws, Plan& p);
// Enqueues the whole computation on `stream`: out_idx / out_dist (m, k).
int run(const float* X, const Plan& p, int squared, int32_t* out_idx, float* out_dist, cudaStream_t stream);

}  // namespace knnx
}  // namespace umapb
