// Shared host/device helpers for libumap_b200: status codes, the thread-local
// error message behind umapb_last_error(), launch checks and workspace carving.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/umap_b200.h"

namespace umapb {

// Records a formatted message for umapb_last_error() and returns `code`.
int set_error(int code, const char* fmt, ...);
// Clears the message (called at the top of every entry point).
void clear_error();

// Converts the last CUDA runtime error (if any) into a status.
int check_cuda(const char* what);

// Adds to the process-wide count of kernels this library has enqueued
// (reported by umapb_kernel_launches()).
void count_launches(int k);

#define UMAPB_REQUIRE(cond, ...)                                          \
  do {                                                                    \
    if (!(cond)) return ::umapb::set_error(UMAPB_ERR_ARG, __VA_ARGS__);   \
  } while (0)

#define UMAPB_CUDA_TRY(expr, what)                                                  \
  do {                                                                              \
    cudaError_t _e = (expr);                                                        \
    if (_e != cudaSuccess)                                                          \
      return ::umapb::set_error(UMAPB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(_e)); \
  } while (0)

#define UMAPB_LAUNCH_CHECK(what)                     \
  do {                                               \
    int _s = ::umapb::check_cuda(what);              \
    if (_s != UMAPB_OK) return _s;                   \
  } while (0)

// Carves aligned sub-buffers out of one caller-owned workspace.  With base ==
// nullptr it only measures, which is how the *_workspace queries are answered.
struct Carver {
  char* base;
  size_t off = 0;
  explicit Carver(void* b) : base(static_cast<char*>(b)) {}
  template <class T>
  T* take(size_t count, size_t align = 256) {
    off = (off + align - 1) / align * align;
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += count * sizeof(T);
    return p;
  }
  size_t bytes() const { return (off + 255) / 256 * 256; }
};

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

int num_sms();  // cached multiProcessorCount of the current device

// Time limit of the bounded device-side waits that take it as a parameter
// (umapb_set_wait_limit_ns; 2 s by default).
unsigned long long wait_limit_ns();

// Device status word values written by kernels with bounded waits.
enum DeviceStatus : int32_t {
  kDevOk = 0,
  kDevTimeoutProducer = 1,
  kDevTimeoutMma = 2,
  kDevTimeoutEpilogue = 3,
  kDevBadLaunch = 4,  // a kernel found its launch shape wrong and did nothing
};

}  // namespace umapb
