// common.cuh -- status handling, per-device context and stream-ordered
// scratch allocation shared by every kernel file of libwetric.
//
// The reference stops the process on any CUDA error (checkCudaErrors,
// tc.cu:46-54); here every failure becomes a status code that travels back
// to the C ABI, with a thread-local message.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <map>
#include <mutex>
#include <string>

#include <nvtx3/nvToolsExt.h>

#include "../../include/wetric.h"

namespace wetric {

// Most row chunks a host-input count copies and counts in turn.
constexpr uint32_t kMaxColChunks = 8;

// ------------------------------------------------------------------ errors

void set_error(int status, const char *fmt, ...);
void clear_error();

struct Status {
  int code = WETRIC_OK;
  bool ok() const { return code == WETRIC_OK; }
};

#define WETRIC_CUDA_TRY(call)                                                 \
  do {                                                                        \
    cudaError_t err_ = (call);                                                \
    if (err_ != cudaSuccess) {                                                \
      int code_ = err_ == cudaErrorMemoryAllocation ? WETRIC_ENOMEM           \
                                                    : WETRIC_ECUDA;           \
      ::wetric::set_error(code_, "%s:%d: %s: %s", __FILE__, __LINE__, #call,  \
                          cudaGetErrorString(err_));                          \
      return code_;                                                           \
    }                                                                         \
  } while (0)

#define WETRIC_TRY(expr)             \
  do {                               \
    int st_ = (expr);                \
    if (st_ != WETRIC_OK) return st_; \
  } while (0)

// Check for a launch error right after a <<<>>> launch.
#define WETRIC_LAUNCH_CHECK() WETRIC_CUDA_TRY(cudaGetLastError())

// ------------------------------------------------------------- context

// One per device: a library stream, an HBM budget, and bookkeeping of the
// bytes this library holds. Scratch comes from the stream-ordered allocator
// (cudaMallocAsync) so repeated calls reuse pool memory without a device
// synchronisation.
struct DeviceContext {
  int device = -1;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // host-to-device copies that overlap
  uint64_t hbm_budget = 0;      // 0 = unlimited
  uint64_t bytes_in_use = 0;
  int sm_count = 0;
  size_t l2_bytes = 0;
  size_t persist_max = 0;       // cudaDevAttrMaxPersistingL2CacheSize
  size_t window_max = 0;        // cudaDevAttrMaxAccessPolicyWindowSize
  std::mutex mu;
  // Batch autotuner results: size/skew bucket -> spread (guarded by mu).
  std::map<uint32_t, uint32_t> spread_table;
  // Pinned staging for pageable host columns: two buffers, each with its
  // own stream, made on first use and held by one count at a time.
  std::mutex stage_mu;
  cudaStream_t stage_stream[2] = {};
  void *stage_buf[2] = {};
  size_t stage_bytes = 0;
};

// Context of `device`, created on first use (thread-safe). Makes `device`
// current on the calling thread.
int get_context(int device, DeviceContext **out);

// Set the HBM budget of a device context (used by fault-injection tests).
int set_budget(int device, uint64_t bytes);

// Stream-ordered device scratch owned by a context.
int dev_alloc(DeviceContext *ctx, cudaStream_t s, size_t bytes, void **p);
void dev_free(DeviceContext *ctx, cudaStream_t s, void *p, size_t bytes);

// RAII holder for one scratch allocation.
template <typename T>
struct Scratch {
  DeviceContext *ctx = nullptr;
  cudaStream_t stream = nullptr;
  T *ptr = nullptr;
  size_t bytes = 0;
  Scratch() = default;
  Scratch(const Scratch &) = delete;
  Scratch &operator=(const Scratch &) = delete;
  int alloc(DeviceContext *c, cudaStream_t s, size_t count) {
    release();
    ctx = c;
    stream = s;
    bytes = count * sizeof(T);
    if (bytes == 0) bytes = 16;
    void *p = nullptr;
    int st = dev_alloc(ctx, stream, bytes, &p);
    if (st != WETRIC_OK) {
      bytes = 0;
      return st;
    }
    ptr = static_cast<T *>(p);
    return WETRIC_OK;
  }
  void release() {
    if (ptr) dev_free(ctx, stream, ptr, bytes);
    ptr = nullptr;
    bytes = 0;
  }
  T *detach() {
    T *p = ptr;
    ptr = nullptr;
    bytes = 0;
    return p;
  }
  ~Scratch() { release(); }
};

// A named NVTX range for the life of the object: the library's stages
// (orientation, the count's prefix / structures / kernels, batches, the
// serving engine) show up by name in a profiler's timeline. NVTX v3 is
// header-only; without a profiler attached the calls do nothing.
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

// ------------------------------------------------------------- helpers

__host__ __device__ __forceinline__ uint64_t ceil_div(uint64_t a, uint64_t b) {
  return (a + b - 1) / b;
}

inline uint32_t bits_for(uint64_t max_value) {
  uint32_t b = 0;
  while (b < 64 && (max_value >> b) != 0) ++b;
  return b;
}

// Kernel-side error word: kernels never trap; they record the first error
// here and the host turns it into a status.
enum DeviceError : uint32_t {
  kDevOk = 0,
  kDevUnsortedRow = 1,
  kDevNotOriented = 2,
  kDevColumnRange = 3,
  kDevDegreeRange = 4,
  kDevRowPtrRange = 5,
};

}  // namespace wetric
