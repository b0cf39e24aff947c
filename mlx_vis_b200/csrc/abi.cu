// Library-wide C-ABI pieces: error reporting, device status readback, cached
// device attributes and TMA descriptor encoding through the driver entry point.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <mutex>

#include "common.cuh"
#include "tc.cuh"

namespace umapb {

static thread_local char g_msg[1024] = {0};

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
  va_end(ap);
  return code;
}

void clear_error() { g_msg[0] = 0; }

int check_cuda(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(UMAPB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return UMAPB_OK;
}

static std::atomic<unsigned long long> g_launches{0};
static std::atomic<unsigned long long> g_wait_limit_ns{2000000000ull};

unsigned long long wait_limit_ns() { return g_wait_limit_ns.load(std::memory_order_relaxed); }

void count_launches(int k) { g_launches.fetch_add((unsigned long long)k, std::memory_order_relaxed); }

int num_sms() {
  int dev = 0;
  cudaGetDevice(&dev);
  static int cache[64] = {0};
  if (dev < 0 || dev >= 64) return 148;
  if (cache[dev] == 0) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    cache[dev] = v > 0 ? v : 148;
  }
  return cache[dev];
}

static PFN_cuTensorMapEncodeTiled_v12000 get_encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

int make_tmap_bf16_2d(CUtensorMap* out, const void* base, uint64_t rows, uint64_t cols, uint64_t pitch_elems,
                      uint32_t box_rows, uint32_t box_cols) {
  auto fn = get_encode_fn();
  if (!fn) return set_error(UMAPB_ERR_CUDA, "cuTensorMapEncodeTiled entry point unavailable");
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0)
    return set_error(UMAPB_ERR_ARG, "TMA base address must be 16-byte aligned");
  if ((pitch_elems * 2) % 16 != 0) return set_error(UMAPB_ERR_ARG, "TMA row pitch must be a multiple of 16 bytes");
  cuuint64_t gdim[2] = {cols, rows};
  cuuint64_t gstride[1] = {pitch_elems * 2};
  cuuint32_t box[2] = {box_cols, box_rows};
  cuuint32_t estride[2] = {1, 1};
  CUresult r = fn(out, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), gdim, gstride, box, estride,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(UMAPB_ERR_CUDA, "cuTensorMapEncodeTiled failed (CUresult %d)", int(r));
  return UMAPB_OK;
}

}  // namespace umapb

extern "C" {

const char* umapb_last_error(void) { return umapb::g_msg; }

int umapb_abi_version(void) { return 1; }

unsigned long long umapb_kernel_launches(void) { return umapb::g_launches.load(std::memory_order_relaxed); }

int umapb_set_wait_limit_ns(unsigned long long ns) {
  umapb::clear_error();
  umapb::g_wait_limit_ns.store(ns ? ns : 2000000000ull, std::memory_order_relaxed);
  return UMAPB_OK;
}

int umapb_read_status(const void* workspace, umapb_stream_t stream) {
  umapb::clear_error();
  if (!workspace) return umapb::set_error(UMAPB_ERR_WORKSPACE, "null workspace");
  int32_t st = 0;
  UMAPB_CUDA_TRY(cudaMemcpyAsync(&st, workspace, sizeof(st), cudaMemcpyDeviceToHost, stream), "status readback");
  UMAPB_CUDA_TRY(cudaStreamSynchronize(stream), "status readback sync");
  if (st != 0)
    return umapb::set_error(UMAPB_ERR_DEVICE,
                            st == umapb::kDevBadLaunch
                                ? "kernel launched with a wrong shape did nothing (code %d); results are invalid"
                                : "device-side wait expired (code %d); results are invalid",
                            int(st));
  return UMAPB_OK;
}

}  // extern "C"
