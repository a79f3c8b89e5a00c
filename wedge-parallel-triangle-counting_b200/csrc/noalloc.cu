// noalloc.cu -- a count entry point that allocates no memory.
//
// Some callers cannot allocate device memory at the time they want a
// count: code that runs inside another framework's memory pool or under a
// hard device-memory quota, real-time or embedded hosts that forbid
// allocation after start-up, and threads that must not take the driver's
// allocation locks. wetric_count_noalloc serves them: it runs the same
// count pipeline as wetric_count_ex on a device-resident oriented CSR, but
// every scratch buffer (active-vertex arrays, prefix sums, tile map,
// bitmap, counters) is carved out of one file-scope device array of
// WETRIC_NOALLOC_SCRATCH_BYTES, which exists on every GPU that loads the
// library until the process exits. No cudaMalloc, cudaMallocAsync,
// cudaFree or allocating library routine is called.
//
// Host code cannot use the array's symbol as a device address (in host
// code it names a host-side stand-in), so the first call on each device
// looks the address up with cudaGetSymbolAddress, with that device
// current, and caches it together with the id of the device's context. A
// later call in another context of that device (after cudaDeviceReset the
// runtime makes a new primary context and loads the module again) sees a
// different id and looks the address up again instead of using a stale
// one. That first call (per device and context) should come before any
// stream capture. Calls share the array and the last call's contents stay in it:
// everything that must start at zero is cleared by each call, and calls
// that overlap on the GPU (two streams, two threads) race on it -- keep
// them ordered.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "../../include/wetric.h"
#include "common.cuh"
#include "count_kernels.cuh"
#include "primitives.cuh"

namespace {

constexpr size_t kNoAllocBytes = WETRIC_NOALLOC_SCRATCH_BYTES;

// The scratch itself: one per device, alive for the life of the process.
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevs = 64;
std::mutex g_noalloc_mu;
// Per device: the scratch address and the id of the context it belongs to.
struct ScratchSlot {
  unsigned long long ctx_id = 0;
  void *ptr = nullptr;
};
ScratchSlot g_noalloc_slot[kMaxDevs];

// Bump allocator over the scratch array (256-byte aligned pieces).
struct Arena {
  unsigned char *base = nullptr;
  size_t used = 0, cap = 0;
  template <typename T>
  T *take(uint64_t count) {
    size_t bytes = (size_t)((count ? count : 1) * sizeof(T));
    bytes = (bytes + 255) & ~(size_t)255;
    if (used + bytes > cap) return nullptr;
    T *p = reinterpret_cast<T *>(base + used);
    used += bytes;
    return p;
  }
};

// Exclusive scan with its block sums taken from the arena (same kernels as
// the allocating scan in primitives.cuh).
template <typename InT, typename OutT>
int scan_in_arena(Arena *ar, cudaStream_t st, const InT *in, OutT *out,
                  uint64_t n) {
  using namespace wetric::prim;
  const uint64_t blocks = n == 0 ? 1 : wetric::ceil_div(n, kScanChunk);
  if (blocks == 1) {
    scan_apply_kernel<InT, OutT><<<1, kScanThreads, 0, st>>>(in, n, out, nullptr);
    WETRIC_LAUNCH_CHECK();
    return WETRIC_OK;
  }
  OutT *sums = ar->take<OutT>(blocks + 1);
  if (!sums) {
    wetric::set_error(WETRIC_ERANGE, "graph too large for the no-allocation scratch");
    return WETRIC_ERANGE;
  }
  scan_reduce_kernel<InT, OutT><<<(unsigned)blocks, kScanThreads, 0, st>>>(in, n, sums);
  WETRIC_LAUNCH_CHECK();
  WETRIC_TRY((scan_in_arena<OutT, OutT>(ar, st, sums, sums, blocks)));
  scan_apply_kernel<InT, OutT><<<(unsigned)blocks, kScanThreads, 0, st>>>(in, n, out, sums);
  WETRIC_LAUNCH_CHECK();
  return WETRIC_OK;
}

// Id of the calling thread's current context: unique for the life of the
// process, so a context made after cudaDeviceReset has a new one. The two
// driver functions are reached through the runtime's entry-point query, so
// the library needs no link to libcuda.
int current_context_id(unsigned long long *id) {
  using GetCurrent = CUresult (*)(CUcontext *);
  using GetId = CUresult (*)(CUcontext, unsigned long long *);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
    cudaGetLastError();
  });
  CUcontext ctx = nullptr;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx ||
      get_id(ctx, id) != CUDA_SUCCESS) {
    wetric::set_error(WETRIC_ECUDA, "cannot identify the current CUDA context");
    return WETRIC_ECUDA;
  }
  return WETRIC_OK;
}

// Address of this device's scratch array, with the device current: looked
// up on the first call in each context of the device and cached with the
// context's id.
int scratch_address(int device, void **out) {
  unsigned long long ctx_id = 0;
  WETRIC_TRY(current_context_id(&ctx_id));
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  ScratchSlot &slot = g_noalloc_slot[device];
  if (!slot.ptr || slot.ctx_id != ctx_id) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      slot = ScratchSlot{};
      wetric::set_error(WETRIC_ECUDA, "cudaGetSymbolAddress of the scratch: %s",
                        cudaGetErrorString(e));
      return WETRIC_ECUDA;
    }
    slot.ptr = p;
    slot.ctx_id = ctx_id;
  }
  *out = slot.ptr;
  return WETRIC_OK;
}

unsigned grid_cap(int sms, uint64_t work) {
  uint64_t g = wetric::ceil_div(work, 256);
  const uint64_t cap = (uint64_t)sms * 8;
  if (g > cap) g = cap;
  return (unsigned)(g ? g : 1);
}

template <typename Off>
int count_noalloc_impl(int device, cudaStream_t st, const Off *rp,
                       const uint32_t *ci, uint64_t n, uint64_t m, uint32_t s,
                       uint32_t a, uint64_t *count) {
  using namespace wetric;
  void *scratch = nullptr;
  WETRIC_TRY(scratch_address(device, &scratch));
  int sms = 0;
  WETRIC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  Arena ar;
  ar.base = static_cast<unsigned char *>(scratch);
  ar.cap = kNoAllocBytes;
  auto too_big = [&]() {
    set_error(WETRIC_ERANGE,
              "graph too large for the no-allocation scratch (%zu bytes)",
              kNoAllocBytes);
    return WETRIC_ERANGE;
  };
  *count = 0;
  if (n == 0) return WETRIC_OK;

  uint32_t *small = ar.take<uint32_t>(4);                   // [0] error
  unsigned long long *acc = ar.take<unsigned long long>(4);  // maxdeg, count, next tile
  uint32_t *active = ar.take<uint32_t>(n);
  uint64_t *pos = ar.take<uint64_t>(n + 1);
  if (!small || !acc || !active || !pos) return too_big();
  WETRIC_CUDA_TRY(cudaMemsetAsync(small, 0, 4 * sizeof(uint32_t), st));
  WETRIC_CUDA_TRY(cudaMemsetAsync(acc, 0, 4 * sizeof(unsigned long long), st));
  k_vertex_wedges<Off><<<grid_cap(sms, n), 256, 0, st>>>(rp, n, m, active, acc, small);
  WETRIC_LAUNCH_CHECK();
  WETRIC_TRY((scan_in_arena<uint32_t, uint64_t>(&ar, st, active, pos, n)));
  uint64_t K = 0;
  unsigned long long maxdeg = 0;
  uint32_t err = 0;
  WETRIC_CUDA_TRY(cudaMemcpyAsync(&K, pos + n, 8, cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(&maxdeg, acc, 8, cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(&err, small, 4, cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  if (err != kDevOk) {
    set_error(WETRIC_EINVAL, "oriented CSR check failed (device code %u)", err);
    return WETRIC_EINVAL;
  }
  if (maxdeg >= kMaxOutDegree) {
    set_error(WETRIC_ERANGE, "max out-degree %llu >= 2^30", maxdeg);
    return WETRIC_ERANGE;
  }
  uint64_t *act_wp = ar.take<uint64_t>(K + 1);
  uint64_t *act_rb = ar.take<uint64_t>(K);
  uint32_t *act_d = ar.take<uint32_t>(K);
  if (!act_wp || !act_rb || !act_d) return too_big();
  if (K > 0) {
    k_compact_active<Off><<<grid_cap(sms, n), 256, 0, st>>>(rp, n, active, pos, act_wp,
                                                           act_rb, act_d);
    WETRIC_LAUNCH_CHECK();
  }
  WETRIC_TRY((scan_in_arena<uint64_t, uint64_t>(&ar, st, act_wp, act_wp, K)));
  uint64_t W = 0;
  WETRIC_CUDA_TRY(cudaMemcpyAsync(&W, act_wp + K, 8, cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  if (W == 0) return WETRIC_OK;

  const uint64_t T = 256ull * s;
  const uint64_t tiles = ceil_div(W, T);
  uint32_t *tile_k = ar.take<uint32_t>(tiles + 1);
  const uint64_t alen = a;
  const uint64_t S = alen * (alen ? alen - 1 : 0) / 2;
  const uint64_t words = ceil_div(S, 32);
  uint32_t *bm = ar.take<uint32_t>(words ? words : 1);
  if (!tile_k || !bm) return too_big();
  k_tile_map<<<grid_cap(sms, tiles + 1), 256, 0, st>>>(act_wp, K, 0, W, T, tiles, tile_k);
  WETRIC_LAUNCH_CHECK();
  const uint64_t bm_first = (n > alen ? n : alen) - alen;
  if (words) {
    WETRIC_CUDA_TRY(cudaMemsetAsync(bm, 0, words * sizeof(uint32_t), st));
    const uint64_t first_row = n - (n < alen ? n : alen);
    k_bitmap<Off><<<grid_cap(sms, (n - first_row) * 32), 256, 0, st>>>(rp, ci, n, first_row,
                                                                      S, bm);
    WETRIC_LAUNCH_CHECK();
  }
  int occ = 0;
  WETRIC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &occ, k_count_rows<Off, false, false>, kWarpsPerBlock * 32, 0));
  uint64_t grid = (uint64_t)sms * (occ < 1 ? 1 : occ);
  const uint64_t need = ceil_div(tiles, kWarpsPerBlock);
  if (grid > need) grid = need;
  k_count_rows<Off, false, false><<<(unsigned)grid, kWarpsPerBlock * 32, 0, st>>>(
      rp, ci, n, act_wp, act_rb, act_d, K, tile_k, tiles, 0, W, T, bm, bm_first, S,
      acc + 2, acc + 1, BatchView{});
  WETRIC_LAUNCH_CHECK();
  unsigned long long tri = 0;
  WETRIC_CUDA_TRY(cudaMemcpyAsync(&tri, acc + 1, 8, cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  *count = tri;
  return WETRIC_OK;
}

}  // namespace

extern "C" int wetric_count_noalloc(const wetric_csr *csr, uint32_t s,
                                    uint32_t a, int device, void *stream,
                                    uint64_t *count) {
  using namespace wetric;
  if (!csr || !count) {
    set_error(WETRIC_EINVAL, "NULL argument");
    return WETRIC_EINVAL;
  }
  if (!(csr->flags & WETRIC_CSR_DEVICE) || !(csr->flags & WETRIC_CSR_ORIENTED)) {
    set_error(WETRIC_EINVAL, "wetric_count_noalloc needs an ORIENTED device CSR");
    return WETRIC_EINVAL;
  }
  if (s == 0 || a % 32 != 0) {
    set_error(WETRIC_EINVAL, "spread must be > 0 and a a multiple of 32");
    return WETRIC_EINVAL;
  }
  if (a > WETRIC_NOALLOC_MAX_BITMAP_LEN || csr->n > WETRIC_NOALLOC_MAX_VERTICES) {
    set_error(WETRIC_ERANGE,
              "wetric_count_noalloc handles n <= %u and a <= %u (got n = %llu, a = %u)",
              (unsigned)WETRIC_NOALLOC_MAX_VERTICES, (unsigned)WETRIC_NOALLOC_MAX_BITMAP_LEN,
              (unsigned long long)csr->n, a);
    return WETRIC_ERANGE;
  }
  if (csr->n > 0 && (!csr->row_ptr || (csr->m > 0 && !csr->col_ind))) {
    set_error(WETRIC_EINVAL, "NULL CSR array");
    return WETRIC_EINVAL;
  }
  int count_dev = 0;
  if (cudaGetDeviceCount(&count_dev) != cudaSuccess || count_dev == 0) {
    cudaGetLastError();
    set_error(WETRIC_ENODEV, "no CUDA device");
    return WETRIC_ENODEV;
  }
  if (device < 0 || device >= count_dev || device >= kMaxDevs) {
    set_error(WETRIC_EINVAL, "device %d out of range", device);
    return WETRIC_EINVAL;
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    set_error(WETRIC_ECUDA, "cudaSetDevice(%d) failed", device);
    return WETRIC_ECUDA;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc;
  if (csr->flags & WETRIC_CSR_OFFSETS32)
    rc = count_noalloc_impl<uint32_t>(device, st, static_cast<const uint32_t *>(csr->row_ptr),
                                      csr->col_ind, csr->n, csr->m, s, a, count);
  else
    rc = count_noalloc_impl<uint64_t>(device, st, static_cast<const uint64_t *>(csr->row_ptr),
                                      csr->col_ind, csr->n, csr->m, s, a, count);
  if (rc == WETRIC_OK) clear_error();
  return rc;
}
