// NNDescent kernels for 32 < k <= 100 (nnd_wide.cu), called by the umapb_nnd_*
// entry points of nndescent.cu when k is above the warp-per-row limit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace umapb {

int nnd_wide_max_k();
int nnd_gather_wide(const float* X, const float* sq, int64_t n, int dd, int32_t* idx, float* dist, int k,
                    int sort_rows, cudaStream_t stream);
int nnd_iteration_wide(const void* Xd, const float* sqd, int dd, int ldx, int half, const int32_t* idx_old,
                       const float* dist_old, const uint8_t* flags_old, const int32_t* rev, int64_t n, int k,
                       int mc_new, int j_nn, int converging, int recompute_cur, int32_t* idx_new, float* dist_new,
                       uint8_t* flags_new, unsigned long long* changed, unsigned long long* evals,
                       cudaStream_t stream);

}  // namespace umapb
