// api.cu -- the extern "C" surface of libwetric (declared in
// include/wetric.h): reference-compatible mirrors of read_graph,
// preprocess, tc_GPU and free_graph, plus wetric_count / wetric_count_ex
// and the device-preprocessing handle.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <omp.h>

#include <mutex>
#include <string>
#include <vector>

#include "batch.cuh"
#include "common.cuh"
#include "count.cuh"
#include "graph_io.h"
#include "preprocess.cuh"

namespace wetric {

// ------------------------------------------------------------------ errors

namespace {
thread_local int t_last_error = WETRIC_OK;
thread_local char t_last_msg[512] = "";
}  // namespace

void set_error(int status, const char *fmt, ...) {
  t_last_error = status;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(t_last_msg, sizeof(t_last_msg), fmt, ap);
  va_end(ap);
}

void clear_error() {
  t_last_error = WETRIC_OK;
  t_last_msg[0] = '\0';
}

// ------------------------------------------------------------- contexts

namespace {
constexpr int kMaxDevices = 64;
constexpr size_t kPoolReserve = 4ull << 30;  // bytes the pool is grown by at set-up
std::mutex g_ctx_mu;
DeviceContext *g_ctx[kMaxDevices] = {};
}  // namespace

int get_context(int device, DeviceContext **out) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    set_error(WETRIC_ENODEV, "no CUDA device (%s)", cudaGetErrorString(e));
    return WETRIC_ENODEV;
  }
  if (device < 0 || device >= count || device >= kMaxDevices) {
    set_error(WETRIC_EINVAL, "device %d out of range (%d devices)", device,
              count);
    return WETRIC_EINVAL;
  }
  WETRIC_CUDA_TRY(cudaSetDevice(device));
  std::lock_guard<std::mutex> lock(g_ctx_mu);
  if (g_ctx[device] == nullptr) {
    DeviceContext *c = new DeviceContext();
    c->device = device;
    cudaError_t err = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (err == cudaSuccess)
      err = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) {
      delete c;
      set_error(WETRIC_ECUDA, "stream create: %s", cudaGetErrorString(err));
      return WETRIC_ECUDA;
    }
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrL2CacheSize, device);
    c->l2_bytes = (size_t)v;
    v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxPersistingL2CacheSize, device);
    c->persist_max = (size_t)v;
    v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxAccessPolicyWindowSize, device);
    c->window_max = (size_t)v;
    // Keep freed scratch in the device's stream-ordered pool between calls
    // instead of returning it to the driver (this process only), and grow
    // the pool once, now, by kPoolReserve (one allocation, freed at once):
    // without it the pool still went to the driver for memory now and then
    // during steady-state counts -- single allocations inside a count took
    // 2-210 ms (R-MAT scale 22, host input: one to three calls in ten at
    // 13-210 ms instead of 12.2), and with it none did. If the reserve
    // cannot be had, the pool grows on demand as before.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t threshold = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
      void *reserve = nullptr;
      if (cudaMallocAsync(&reserve, kPoolReserve, c->stream) == cudaSuccess) {
        cudaFreeAsync(reserve, c->stream);
        cudaStreamSynchronize(c->stream);
      }
    }
    cudaGetLastError();
    g_ctx[device] = c;
  }
  *out = g_ctx[device];
  return WETRIC_OK;
}

int set_budget(int device, uint64_t bytes) {
  DeviceContext *c = nullptr;
  WETRIC_TRY(get_context(device, &c));
  std::lock_guard<std::mutex> lock(c->mu);
  c->hbm_budget = bytes;
  return WETRIC_OK;
}

int dev_alloc(DeviceContext *ctx, cudaStream_t s, size_t bytes, void **p) {
  {
    std::lock_guard<std::mutex> lock(ctx->mu);
    if (ctx->hbm_budget && ctx->bytes_in_use + bytes > ctx->hbm_budget) {
      set_error(WETRIC_ENOMEM,
                "HBM budget exceeded: %llu in use + %llu requested > %llu",
                (unsigned long long)ctx->bytes_in_use,
                (unsigned long long)bytes,
                (unsigned long long)ctx->hbm_budget);
      return WETRIC_ENOMEM;
    }
    ctx->bytes_in_use += bytes;
  }
  cudaError_t e = cudaMallocAsync(p, bytes, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->bytes_in_use -= bytes;
    *p = nullptr;
    const int code =
        e == cudaErrorMemoryAllocation ? WETRIC_ENOMEM : WETRIC_ECUDA;
    set_error(code, "device allocation of %llu bytes: %s",
              (unsigned long long)bytes, cudaGetErrorString(e));
    return code;
  }
  return WETRIC_OK;
}

void dev_free(DeviceContext *ctx, cudaStream_t s, void *p, size_t bytes) {
  if (!p) return;
  cudaFreeAsync(p, s);
  std::lock_guard<std::mutex> lock(ctx->mu);
  ctx->bytes_in_use -= bytes;
}

}  // namespace wetric

using namespace wetric;

struct wetric_oriented_s {
  DeviceCsr csr;
};

struct wetric_batch_s {
  Batch batch;
};

namespace {

// Records the status of a failing call (so wetric_last_error() works for
// the sentinel-returning entry points) and passes it through.
int finish(int st) {
  if (st == WETRIC_OK) clear_error();
  return st;
}

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  ~Timer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
  int start(cudaStream_t s) {
    WETRIC_CUDA_TRY(cudaEventCreate(&a));
    WETRIC_CUDA_TRY(cudaEventCreate(&b));
    WETRIC_CUDA_TRY(cudaEventRecord(a, s));
    return WETRIC_OK;
  }
  int stop(cudaStream_t s, double *ms) {
    WETRIC_CUDA_TRY(cudaEventRecord(b, s));
    WETRIC_CUDA_TRY(cudaEventSynchronize(b));
    float f = 0;
    WETRIC_CUDA_TRY(cudaEventElapsedTime(&f, a, b));
    *ms = f;
    return WETRIC_OK;
  }
};

// Host-input counts of at least this many columns copy them in row chunks.
constexpr uint64_t kChunkMinColumns = 1ull << 22;

uint64_t host_offset(const void *row_ptr, bool off32, uint64_t v) {
  return off32 ? static_cast<const uint32_t *>(row_ptr)[v]
               : static_cast<const uint64_t *>(row_ptr)[v];
}

// Row chunks of a host CSR, highest rows first, growing geometrically:
// the top 1/64 of the columns, then up to the top 1/16, 1/8, 1/4, 1/2, 3/4
// and the rest. The highest rows hold the most wedges per column (on R-MAT
// scale 22 the top 1/8 of the columns carries 37% of the wedges), so a
// small first chunk starts the count early and the larger ones still
// arrive before the count reaches them. chunk_lo[i] is the first row of
// chunk i and the last one is 0. Returns the number of chunks, or 0 when
// the offsets at the boundaries do not rise from 0 to m (the count's own
// row checks then report the CSR; its columns are copied whole).
constexpr uint32_t kChunkTop64ths[] = {1, 4, 8, 16, 32, 48};  // of 64
static_assert(sizeof(kChunkTop64ths) / sizeof(uint32_t) < kMaxColChunks,
              "chunk table fits the count's chunk limit");
uint32_t column_chunks(const void *row_ptr, bool off32, uint64_t n, uint64_t m,
                       uint64_t *chunk_lo) {
  if (host_offset(row_ptr, off32, 0) != 0 || host_offset(row_ptr, off32, n) != m)
    return 0;
  uint32_t c = 0;
  uint64_t prev = n;
  for (uint32_t top : kChunkTop64ths) {
    // first row whose columns start at or after the top top/64 of them
    const uint64_t target = m - m / 64 * top - (m % 64) * top / 64;
    uint64_t lo = 0, hi = prev;
    while (lo < hi) {
      const uint64_t mid = lo + (hi - lo) / 2;
      if (host_offset(row_ptr, off32, mid) >= target) hi = mid;
      else lo = mid + 1;
    }
    if (lo > 0 && lo < prev) {
      chunk_lo[c++] = lo;
      prev = lo;
    }
  }
  chunk_lo[c++] = 0;
  // offsets at the boundaries must not decrease (the copy ranges)
  uint64_t hi_off = m;
  for (uint32_t i = 0; i < c; ++i) {
    const uint64_t lo_off = host_offset(row_ptr, off32, chunk_lo[i]);
    if (lo_off > hi_off) return 0;
    hi_off = lo_off;
  }
  return c;
}

// ------------------------------------------- pinned staging of host columns
//
// A cudaMemcpyAsync from pageable memory is staged by the driver and does
// not return before the data is staged, so the count's host thread would
// copy every column before it could launch any chunk's kernels. For
// pageable columns the library stages them itself instead: pieces of at
// most kStageBytes alternate between two pinned buffers, each with its own
// stream; on each stream a host function copies the piece into the buffer
// (all host threads, OpenMP) and a DMA moves it to the device. The copy of
// piece p + 1 runs while piece p's DMA is in flight, a buffer is reused
// only after its previous DMA (stream order), and nothing blocks the
// count's thread.
constexpr size_t kStageBytes = 16ull << 20;

bool host_pageable(const void *p) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return at.type == cudaMemoryTypeUnregistered;
}

// The context's two pinned buffers and streams (made once, under stage_mu).
int stage_buffers(DeviceContext *ctx) {
  if (ctx->stage_buf[0]) return WETRIC_OK;
  for (int i = 0; i < 2; ++i) {
    WETRIC_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->stage_stream[i], cudaStreamNonBlocking));
    WETRIC_CUDA_TRY(cudaHostAlloc(&ctx->stage_buf[i], kStageBytes, cudaHostAllocDefault));
  }
  ctx->stage_bytes = kStageBytes;
  return WETRIC_OK;
}

struct StagePiece {
  const void *src = nullptr;
  void *dst = nullptr;
  size_t bytes = 0;
};

void CUDART_CB stage_copy(void *p) {
  const StagePiece *pc = static_cast<const StagePiece *>(p);
  const size_t block = 1ull << 20;
  const int64_t blocks = (int64_t)((pc->bytes + block - 1) / block);
  const char *src = static_cast<const char *>(pc->src);
  char *dst = static_cast<char *>(pc->dst);
#pragma omp parallel for schedule(static) num_threads(omp_get_num_procs() < 16 ? omp_get_num_procs() : 16)
  for (int64_t b = 0; b < blocks; ++b) {
    const size_t o = (size_t)b * block;
    memcpy(dst + o, src + o, o + block <= pc->bytes ? block : pc->bytes - o);
  }
}

int count_ex_impl(const wetric_csr *csr, const wetric_opts *o,
                  uint64_t *count, wetric_stats *stats) {
  NvtxRange nvtx_("wetric_count_ex");
  if (!csr || !o || !count) {
    set_error(WETRIC_EINVAL, "NULL argument");
    return WETRIC_EINVAL;
  }
  if (o->spread == 0) {
    set_error(WETRIC_EINVAL, "spread must be > 0");
    return WETRIC_EINVAL;
  }
  if (o->bitmap_len % 32 != 0) {
    set_error(WETRIC_EINVAL, "bitmap length %u is not a multiple of 32",
              o->bitmap_len);
    return WETRIC_EINVAL;
  }
  const uint32_t f = csr->flags;
  const bool on_device = (f & WETRIC_CSR_DEVICE) != 0;
  const bool off32 = (f & WETRIC_CSR_OFFSETS32) != 0;
  const bool symmetric = (f & WETRIC_CSR_SYMMETRIC) != 0;
  if ((f & WETRIC_CSR_ORIENTED) && symmetric) {
    set_error(WETRIC_EINVAL, "CSR cannot be both ORIENTED and SYMMETRIC");
    return WETRIC_EINVAL;
  }
  if (csr->n >= (1ull << 32)) {
    set_error(WETRIC_ERANGE, "n = %llu exceeds 2^32 - 1",
              (unsigned long long)csr->n);
    return WETRIC_ERANGE;
  }
  if (off32 && csr->m >= (1ull << 32)) {
    set_error(WETRIC_ERANGE, "u32 offsets with m >= 2^32");
    return WETRIC_ERANGE;
  }
  if (csr->n > 0 && (!csr->row_ptr || (csr->m > 0 && !csr->col_ind))) {
    set_error(WETRIC_EINVAL, "NULL CSR array");
    return WETRIC_EINVAL;
  }
  DeviceContext *ctx = nullptr;
  WETRIC_TRY(get_context(o->device, &ctx));
  cudaStream_t st = o->stream ? static_cast<cudaStream_t>(o->stream) : ctx->stream;
  const uint64_t n = csr->n, m = csr->m;
  wetric_stats s = {};
  s.spread = o->spread;
  s.bitmap_len = o->bitmap_len;

  // 1. Device copies of the caller's arrays (host input). For an oriented
  //    CSR the columns are copied on the context's copy stream while the
  //    count works on the row offsets -- for a large graph in row chunks,
  //    highest rows first, so the count of the top vertices starts while
  //    the rows below them are still copying.
  Scratch<uint8_t> d_rp;
  Scratch<uint32_t> d_ci;
  // declared after the buffers, so it is destroyed first: its wait orders
  // their stream-ordered frees after the column copy
  struct CopyEvents {
    cudaEvent_t start = nullptr, rp_done = nullptr, ci_done = nullptr;
    cudaEvent_t ci_start = nullptr;  // chunked copies: when they were issued
    cudaEvent_t chunk[kMaxColChunks] = {};
    cudaStream_t st = nullptr;
    bool ci_recorded = false;
    // chunked copies, issued from the count once its read-back is done
    const void *h_rp = nullptr;
    const uint32_t *h_ci = nullptr;
    uint32_t *d_ci = nullptr;
    bool off32 = false;
    uint64_t n = 0;
    uint32_t nchunks = 0;
    uint64_t chunk_lo[kMaxColChunks] = {};
    cudaStream_t copy = nullptr;
    // pageable columns: staged through the context's pinned buffers
    DeviceContext *stage_ctx = nullptr;
    std::unique_lock<std::mutex> stage_lock;
    std::vector<StagePiece> pieces;
    cudaEvent_t join = nullptr;
    ~CopyEvents() {
      // the column buffer is freed on `st`: order that after the copy
      if (ci_done && ci_recorded && st) cudaStreamWaitEvent(st, ci_done, 0);
      // staged pieces: their host functions read `pieces`, so wait for them
      if (stage_ctx) {
        for (cudaStream_t x : stage_ctx->stage_stream) cudaStreamSynchronize(x);
        cudaGetLastError();
      }
      for (cudaEvent_t e : {start, rp_done, ci_done, ci_start, join})
        if (e) cudaEventDestroy(e);
      for (cudaEvent_t e : chunk)
        if (e) cudaEventDestroy(e);
    }
    // Marks the end of every column copy queued so far on stream `on`, so
    // the destructor orders the buffer's free after them. If the event
    // cannot be recorded, waits for the stream instead.
    int mark_copies_done(cudaStream_t on) {
      const cudaError_t e = cudaEventRecord(ci_done, on);
      if (e == cudaSuccess) {
        ci_recorded = true;
        return WETRIC_OK;
      }
      cudaGetLastError();
      cudaStreamSynchronize(on);
      cudaGetLastError();
      wetric::set_error(WETRIC_ECUDA, "cudaEventRecord after the column copies: %s",
                        cudaGetErrorString(e));
      return WETRIC_ECUDA;
    }
    // rows [chunk_lo[i], chunk_lo[i - 1]), highest first; the offsets at
    // the boundaries were checked to rise from 0 to m
    int issue_chunks() {
      WETRIC_CUDA_TRY(cudaEventRecord(ci_start, copy));
      if (stage_ctx) return issue_staged();
      for (uint32_t i = 0; i < nchunks; ++i) {
        const uint64_t c0 = host_offset(h_rp, off32, chunk_lo[i]);
        const uint64_t c1 = host_offset(h_rp, off32, i ? chunk_lo[i - 1] : n);
        if (c1 > c0)
          WETRIC_CUDA_TRY(cudaMemcpyAsync(d_ci + c0, h_ci + c0, (c1 - c0) * sizeof(uint32_t),
                                          cudaMemcpyHostToDevice, copy));
        WETRIC_CUDA_TRY(cudaEventRecord(chunk[i], copy));
      }
      return WETRIC_OK;
    }
    // The same chunks through the pinned buffers: piece q on buffer and
    // stream q % 2; chunk i's event on `copy` after both streams reach the
    // end of its pieces.
    int issue_staged() {
      cudaStream_t *xs = stage_ctx->stage_stream;
      for (cudaStream_t x : {xs[0], xs[1]}) WETRIC_CUDA_TRY(cudaStreamWaitEvent(x, ci_start, 0));
      const size_t piece_cols = stage_ctx->stage_bytes / sizeof(uint32_t);
      size_t total = 0;
      for (uint32_t i = 0; i < nchunks; ++i) {
        const uint64_t c0 = host_offset(h_rp, off32, chunk_lo[i]);
        const uint64_t c1 = host_offset(h_rp, off32, i ? chunk_lo[i - 1] : n);
        total += c1 > c0 ? ceil_div(c1 - c0, piece_cols) : 0;
      }
      pieces.assign(total, StagePiece{});  // no reallocation below: host
      size_t q = 0;                        // functions hold pointers into it
      for (uint32_t i = 0; i < nchunks; ++i) {
        const uint64_t c0 = host_offset(h_rp, off32, chunk_lo[i]);
        const uint64_t c1 = host_offset(h_rp, off32, i ? chunk_lo[i - 1] : n);
        for (uint64_t a = c0; a < c1; a += piece_cols, ++q) {
          const uint64_t b = a + piece_cols < c1 ? a + piece_cols : c1;
          StagePiece &pc = pieces[q];
          pc.src = h_ci + a;
          pc.dst = stage_ctx->stage_buf[q & 1];
          pc.bytes = (b - a) * sizeof(uint32_t);
          WETRIC_CUDA_TRY(cudaLaunchHostFunc(xs[q & 1], stage_copy, &pc));
          WETRIC_CUDA_TRY(cudaMemcpyAsync(d_ci + a, pc.dst, pc.bytes, cudaMemcpyHostToDevice,
                                          xs[q & 1]));
        }
        WETRIC_CUDA_TRY(cudaEventRecord(join, xs[0]));
        WETRIC_CUDA_TRY(cudaStreamWaitEvent(copy, join, 0));
        WETRIC_CUDA_TRY(cudaEventRecord(join, xs[1]));
        WETRIC_CUDA_TRY(cudaStreamWaitEvent(copy, join, 0));
        WETRIC_CUDA_TRY(cudaEventRecord(chunk[i], copy));
      }
      return WETRIC_OK;
    }
    // Issues the chunk copies; on success and on failure alike, ci_done
    // then follows every copy that was queued.
    static int issue(void *p) {
      CopyEvents *c = static_cast<CopyEvents *>(p);
      const int rc = c->issue_chunks();
      const int done = c->mark_copies_done(c->copy);
      return rc != WETRIC_OK ? rc : done;
    }
  } cev;
  uint32_t nchunks = 0;
  uint64_t chunk_lo[kMaxColChunks] = {};
  const void *rp = csr->row_ptr;
  const uint32_t *ci = csr->col_ind;
  cudaEvent_t ci_ready = nullptr;
  const size_t rp_bytes = (n + 1) * (off32 ? sizeof(uint32_t) : sizeof(uint64_t));
  if (!on_device && n > 0) {
    WETRIC_TRY(d_rp.alloc(ctx, st, rp_bytes));
    WETRIC_TRY(d_ci.alloc(ctx, st, m));
    WETRIC_CUDA_TRY(cudaEventCreate(&cev.start));
    WETRIC_CUDA_TRY(cudaEventCreate(&cev.rp_done));
    WETRIC_CUDA_TRY(cudaEventRecord(cev.start, st));
    WETRIC_CUDA_TRY(cudaMemcpyAsync(d_rp.ptr, csr->row_ptr, rp_bytes,
                                    cudaMemcpyHostToDevice, st));
    if (m > 0 && !symmetric) {
      cev.st = st;
      // the copy stream starts after the allocation (stream-ordered on st)
      WETRIC_CUDA_TRY(cudaStreamWaitEvent(ctx->copy_stream, cev.start, 0));
      if (!o->validate && m >= kChunkMinColumns)
        nchunks = column_chunks(csr->row_ptr, off32, n, m, chunk_lo);
      WETRIC_CUDA_TRY(cudaEventCreateWithFlags(&cev.ci_done, cudaEventDefault));
      if (nchunks > 1) {
        // issued by the count after its read-back (CountArgs::issue_copies)
        WETRIC_CUDA_TRY(cudaEventCreateWithFlags(&cev.ci_start, cudaEventDefault));
        for (uint32_t i = 0; i < nchunks; ++i) {
          WETRIC_CUDA_TRY(cudaEventCreateWithFlags(&cev.chunk[i], cudaEventDisableTiming));
          cev.chunk_lo[i] = chunk_lo[i];
        }
        cev.h_rp = csr->row_ptr;
        cev.h_ci = csr->col_ind;
        cev.d_ci = d_ci.ptr;
        cev.off32 = off32;
        cev.n = n;
        cev.nchunks = nchunks;
        cev.copy = ctx->copy_stream;
        // Pageable columns go through the pinned staging buffers when this
        // count can have them (another count holding them copies directly).
        if (host_pageable(csr->col_ind)) {
          std::unique_lock<std::mutex> lk(ctx->stage_mu, std::try_to_lock);
          if (lk.owns_lock() && stage_buffers(ctx) == WETRIC_OK &&
              cudaEventCreateWithFlags(&cev.join, cudaEventDisableTiming) == cudaSuccess) {
            cev.stage_ctx = ctx;
            cev.stage_lock = std::move(lk);
          }
          cudaGetLastError();
          clear_error();
        }
      } else {
        nchunks = 0;
        WETRIC_CUDA_TRY(cudaMemcpyAsync(d_ci.ptr, csr->col_ind, m * sizeof(uint32_t),
                                        cudaMemcpyHostToDevice, ctx->copy_stream));
        WETRIC_TRY(cev.mark_copies_done(ctx->copy_stream));
        ci_ready = cev.ci_done;
      }
    } else if (m > 0) {
      WETRIC_CUDA_TRY(cudaMemcpyAsync(d_ci.ptr, csr->col_ind, m * sizeof(uint32_t),
                                      cudaMemcpyHostToDevice, st));
    }
    WETRIC_CUDA_TRY(cudaEventRecord(cev.rp_done, st));
    rp = d_rp.ptr;
    ci = d_ci.ptr;
  }

  // 2. Orientation on the device for SYMMETRIC input.
  DeviceCsr oriented;
  uint64_t cn = n, cm = m;
  bool c_off32 = off32;
  if (symmetric && n > 0) {
    Timer tm;
    WETRIC_TRY(tm.start(st));
    const uint64_t *rp64 = static_cast<const uint64_t *>(rp);
    Scratch<uint64_t> wide;
    if (off32) {
      WETRIC_TRY(wide.alloc(ctx, st, n + 1));
      WETRIC_TRY(widen_offsets(ctx, st, static_cast<const uint32_t *>(rp), n,
                               wide.ptr));
      rp64 = wide.ptr;
    }
    WETRIC_TRY(orient_csr(ctx, st, rp64, ci, n, m, &oriented));
    WETRIC_TRY(tm.stop(st, &s.prep_ms));
    rp = oriented.row_ptr;
    ci = oriented.col_ind;
    cn = oriented.n;
    cm = oriented.m;
    c_off32 = false;
  }

  // 3. u32 row offsets for the count when m < 2^32 (halves the offset
  //    bytes of every edge check).
  Scratch<uint32_t> narrow;
  if (!c_off32 && cm < (1ull << 32) && cn > 0 &&
      !(o->opt_flags & WETRIC_OPT_KEEP_U64_OFFSETS)) {
    WETRIC_TRY(narrow.alloc(ctx, st, cn + 1));
    WETRIC_TRY(narrow_offsets(ctx, st, static_cast<const uint64_t *>(rp), cn,
                              narrow.ptr));
    rp = narrow.ptr;
    c_off32 = true;
  }

  CountArgs a;
  a.n = cn;
  a.m = cm;
  a.row_ptr = rp;
  a.offsets32 = c_off32;
  a.col_ind = ci;
  a.spread = o->spread;
  a.bitmap_len = o->bitmap_len;
  a.block = o->block;
  a.wedge_begin = o->wedge_begin;
  a.wedge_end = o->wedge_end;
  a.validate = o->validate != 0;
  a.l2_persist = o->l2_persist != 0;
  a.kernel = o->kernel;
  a.core_len = o->core_len;
  a.shell_len = o->shell_len;
  a.persistent = !(o->opt_flags & WETRIC_OPT_ONE_PASS);
  a.pair_streams = !(o->opt_flags & WETRIC_OPT_NO_PAIR_STREAMS);
  a.ci_ready = ci_ready;
  if (nchunks > 1) {
    a.col_chunks = nchunks;
    for (uint32_t i = 0; i < nchunks; ++i) {
      a.chunk_lo[i] = chunk_lo[i];
      a.chunk_ready[i] = cev.chunk[i];
    }
    a.issue_copies = &CopyEvents::issue;
    a.issue_ctx = &cev;
  }
  if (o->kernel > 8) {
    set_error(WETRIC_EINVAL, "unknown count kernel %u", o->kernel);
    return WETRIC_EINVAL;
  }
  CountResult r;
  WETRIC_TRY(count_oriented(ctx, st, a, &r));
  if (cev.start) {
    // copy time: from the first copy to the later of the two copies' ends;
    // chunked columns: the row offsets' copy plus the columns' copies
    float f = 0, g = 0;
    WETRIC_CUDA_TRY(cudaEventSynchronize(cev.rp_done));
    WETRIC_CUDA_TRY(cudaEventElapsedTime(&f, cev.start, cev.rp_done));
    if (cev.ci_done && cev.ci_recorded) {
      WETRIC_CUDA_TRY(cudaEventSynchronize(cev.ci_done));
      if (cev.ci_start) {
        WETRIC_CUDA_TRY(cudaEventElapsedTime(&g, cev.ci_start, cev.ci_done));
        g += f;
      } else {
        WETRIC_CUDA_TRY(cudaEventElapsedTime(&g, cev.start, cev.ci_done));
      }
    }
    s.copy_ms = f > g ? f : g;
  }
  *count = r.triangles;
  s.exec_ms = r.exec_ms;
  s.count_ms = r.count_ms;
  s.n = cn;
  s.m = cm;
  s.wedges = r.wedges;
  s.wedges_counted = r.wedges_counted;
  s.max_out_degree = r.max_out_degree;
  s.block = r.block;
  s.grid = r.grid;
  s.launches = r.launches;
  s.core_len = r.core_len;
  s.core_wedges = r.core_wedges;
  s.core_ms = r.core_ms;
  s.shell_len = r.shell_len;
  s.shell_wedges = r.shell_wedges;
  s.shell_ms = r.shell_ms;
  s.pair_rows = r.pair_rows;
  s.pair_wedges = r.pair_wedges;
  s.pair_ms = r.pair_ms;
  if (stats) *stats = s;
  return WETRIC_OK;
}

uint64_t tc_gpu_common(uint64_t n, uint64_t m, const void *rp, bool off32,
                       const uint32_t *ci, uint32_t spread, uint32_t a,
                       wetric_gpu_time *t) {
  wetric_csr csr;
  csr.n = n;
  csr.m = m;
  csr.row_ptr = rp;
  csr.col_ind = ci;
  csr.flags = WETRIC_CSR_ORIENTED | (off32 ? WETRIC_CSR_OFFSETS32 : 0u);
  wetric_opts o;
  wetric_opts_init(&o);
  o.spread = spread;
  o.bitmap_len = a;
  uint64_t count = 0;
  wetric_stats s;
  const int st = finish(count_ex_impl(&csr, &o, &count, &s));
  if (st != WETRIC_OK) return UINT64_MAX;
  if (t) {
    t->copy += s.copy_ms;
    t->exec += s.exec_ms;
  }
  return count;
}

// Host pairs -> device -> symmetric CSR (device) -> host arrays.
int read_graph_impl(const char *filename, int mm, int zero_indexed,
                    DeviceContext **ctx_out, DeviceCsr *sym) {
  if (!filename) {
    set_error(WETRIC_EINVAL, "NULL filename");
    return WETRIC_EINVAL;
  }
  std::vector<uint32_t> src, dst;
  uint64_t n = 0;
  std::string msg;
  const int st = parse_edge_file(filename, mm != 0, zero_indexed != 0, &src,
                                 &dst, &n, &msg);
  if (st != WETRIC_OK) {
    set_error(st, "%s", msg.c_str());
    return st;
  }
  DeviceContext *ctx = nullptr;
  WETRIC_TRY(get_context(0, &ctx));
  cudaStream_t s = ctx->stream;
  const uint64_t P = src.size();
  Scratch<uint32_t> ds, dd;
  WETRIC_TRY(ds.alloc(ctx, s, P));
  WETRIC_TRY(dd.alloc(ctx, s, P));
  if (P) {
    WETRIC_CUDA_TRY(cudaMemcpyAsync(ds.ptr, src.data(), P * 4,
                                    cudaMemcpyHostToDevice, s));
    WETRIC_CUDA_TRY(cudaMemcpyAsync(dd.ptr, dst.data(), P * 4,
                                    cudaMemcpyHostToDevice, s));
  }
  WETRIC_TRY(symmetric_from_pairs(ctx, s, ds.ptr, dd.ptr, P, n, sym));
  *ctx_out = ctx;
  return WETRIC_OK;
}

template <typename G, typename Off>
G *download_graph(DeviceContext *ctx, const DeviceCsr &c, int *st) {
  cudaStream_t s = ctx->stream;
  G *g = (G *)calloc(1, sizeof(G));
  Off *rp = (Off *)malloc((c.n + 1) * sizeof(Off));
  uint32_t *ci = (uint32_t *)malloc((c.m ? c.m : 1) * sizeof(uint32_t));
  uint64_t *tmp = (uint64_t *)malloc((c.n + 1) * sizeof(uint64_t));
  if (!g || !rp || !ci || !tmp) {
    free(g);
    free(rp);
    free(ci);
    free(tmp);
    set_error(WETRIC_ENOMEM, "host allocation failed");
    *st = WETRIC_ENOMEM;
    return nullptr;
  }
  cudaError_t e = cudaMemcpyAsync(tmp, c.row_ptr, (c.n + 1) * sizeof(uint64_t),
                                  cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && c.m)
    e = cudaMemcpyAsync(ci, c.col_ind, c.m * sizeof(uint32_t),
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    free(g);
    free(rp);
    free(ci);
    free(tmp);
    set_error(WETRIC_ECUDA, "download: %s", cudaGetErrorString(e));
    *st = WETRIC_ECUDA;
    return nullptr;
  }
  for (uint64_t i = 0; i <= c.n; ++i) rp[i] = (Off)tmp[i];
  free(tmp);
  g->numVertices = (uint32_t)c.n;
  g->numEdges = (decltype(g->numEdges))c.m;
  g->rowPtr = rp;
  g->colInd = ci;
  *st = WETRIC_OK;
  return g;
}

template <typename G, typename Off>
G *preprocess_impl(const G *in, int *st) {
  if (!in || (in->numVertices > 0 && !in->rowPtr)) {
    set_error(WETRIC_EINVAL, "NULL graph");
    *st = WETRIC_EINVAL;
    return nullptr;
  }
  DeviceContext *ctx = nullptr;
  if ((*st = get_context(0, &ctx)) != WETRIC_OK) return nullptr;
  cudaStream_t s = ctx->stream;
  const uint64_t n = in->numVertices, m = in->numEdges;
  Scratch<Off> drp_in;
  Scratch<uint64_t> drp;
  Scratch<uint32_t> dci;
  DeviceCsr out;
  auto run = [&]() -> int {
    WETRIC_TRY(drp_in.alloc(ctx, s, n + 1));
    WETRIC_TRY(drp.alloc(ctx, s, n + 1));
    WETRIC_TRY(dci.alloc(ctx, s, m));
    WETRIC_CUDA_TRY(cudaMemcpyAsync(drp_in.ptr, in->rowPtr, (n + 1) * sizeof(Off),
                                    cudaMemcpyHostToDevice, s));
    if (m)
      WETRIC_CUDA_TRY(cudaMemcpyAsync(dci.ptr, in->colInd, m * 4,
                                      cudaMemcpyHostToDevice, s));
    if (sizeof(Off) == 4) {
      WETRIC_TRY(widen_offsets(ctx, s, (const uint32_t *)drp_in.ptr, n, drp.ptr));
    } else {
      WETRIC_CUDA_TRY(cudaMemcpyAsync(drp.ptr, drp_in.ptr, (n + 1) * 8,
                                      cudaMemcpyDeviceToDevice, s));
    }
    WETRIC_TRY(orient_csr(ctx, s, drp.ptr, dci.ptr, n, m, &out));
    return WETRIC_OK;
  };
  if (n == 0) {
    set_error(WETRIC_EINVAL, "graph without vertices");
    *st = WETRIC_EINVAL;
    return nullptr;
  }
  if ((*st = run()) != WETRIC_OK) return nullptr;
  return download_graph<G, Off>(ctx, out, st);
}

}  // namespace

extern "C" {

int wetric_last_error(void) { return t_last_error; }

const char *wetric_last_error_message(void) { return t_last_msg; }

const char *wetric_strerror(int status) {
  switch (status) {
    case WETRIC_OK: return "ok";
    case WETRIC_EINVAL: return "invalid argument";
    case WETRIC_ENOMEM: return "out of memory or over the HBM budget";
    case WETRIC_ETIMEDOUT: return "bounded device wait timed out";
    case WETRIC_ECUDA: return "CUDA runtime error";
    case WETRIC_ERANGE: return "size out of supported range";
    case WETRIC_EIO: return "graph file unreadable or malformed";
    case WETRIC_ENODEV: return "no CUDA device";
    case WETRIC_EBUSY: return "busy";
    default: return "unknown status";
  }
}

void wetric_opts_init(wetric_opts *o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->spread = 5;
  o->bitmap_len = 8192;
  o->device = 0;
}

int wetric_set_hbm_budget(int device, uint64_t bytes) {
  return finish(set_budget(device, bytes));
}

uint64_t wetric_count(const wetric_csr *csr, uint32_t s, uint32_t a) {
  wetric_opts o;
  wetric_opts_init(&o);
  o.spread = s;
  o.bitmap_len = a;
  uint64_t c = 0;
  if (finish(count_ex_impl(csr, &o, &c, nullptr)) != WETRIC_OK) return UINT64_MAX;
  return c;
}

int wetric_count_ex(const wetric_csr *csr, const wetric_opts *opts,
                    uint64_t *count, wetric_stats *stats) {
  wetric_opts o;
  if (opts) {
    o = *opts;
  } else {
    wetric_opts_init(&o);
  }
  return finish(count_ex_impl(csr, &o, count, stats));
}

uint64_t wetric_tc_gpu(const wetric_graph *g, uint32_t spread, uint32_t a,
                       wetric_gpu_time *t) {
  if (!g) {
    set_error(WETRIC_EINVAL, "NULL graph");
    return UINT64_MAX;
  }
  return tc_gpu_common(g->numVertices, g->numEdges, g->rowPtr, true,
                       g->colInd, spread, a, t);
}

uint64_t wetric_tc_gpu_big(const wetric_big_graph *g, uint32_t spread,
                           uint32_t a, wetric_gpu_time *t) {
  if (!g) {
    set_error(WETRIC_EINVAL, "NULL graph");
    return UINT64_MAX;
  }
  return tc_gpu_common(g->numVertices, g->numEdges, g->rowPtr, false,
                       g->colInd, spread, a, t);
}

wetric_graph *wetric_read_graph(const char *filename, int mm, int zero_indexed,
                                int preprocess_style) {
  (void)preprocess_style;
  DeviceContext *ctx = nullptr;
  DeviceCsr sym;
  int st = read_graph_impl(filename, mm, zero_indexed, &ctx, &sym);
  if (st != WETRIC_OK) return nullptr;
  if (sym.m >= (1ull << 32)) {
    set_error(WETRIC_ERANGE, "%llu directed edges do not fit u32 offsets; "
              "use wetric_read_big_graph", (unsigned long long)sym.m);
    return nullptr;
  }
  wetric_graph *g = download_graph<wetric_graph, uint32_t>(ctx, sym, &st);
  if (g) clear_error();
  return g;
}

wetric_big_graph *wetric_read_big_graph(const char *filename, int mm,
                                        int zero_indexed,
                                        int preprocess_style) {
  (void)preprocess_style;
  DeviceContext *ctx = nullptr;
  DeviceCsr sym;
  int st = read_graph_impl(filename, mm, zero_indexed, &ctx, &sym);
  if (st != WETRIC_OK) return nullptr;
  wetric_big_graph *g = download_graph<wetric_big_graph, uint64_t>(ctx, sym, &st);
  if (g) clear_error();
  return g;
}

wetric_graph *wetric_preprocess(const wetric_graph *g, int preprocess_style) {
  (void)preprocess_style;
  int st = WETRIC_OK;
  wetric_graph *r = preprocess_impl<wetric_graph, uint32_t>(g, &st);
  if (r) clear_error();
  return r;
}

wetric_big_graph *wetric_preprocess_big(const wetric_big_graph *g,
                                        int preprocess_style) {
  (void)preprocess_style;
  int st = WETRIC_OK;
  wetric_big_graph *r = preprocess_impl<wetric_big_graph, uint64_t>(g, &st);
  if (r) clear_error();
  return r;
}

void wetric_free_graph(wetric_graph *g) {
  if (!g) return;
  free(g->rowPtr);
  free(g->colInd);
  free(g);
}

void wetric_free_big_graph(wetric_big_graph *g) {
  if (!g) return;
  free(g->rowPtr);
  free(g->colInd);
  free(g);
}

int wetric_wedge_total(const wetric_csr *csr, int device, uint64_t *wedges,
                       uint64_t *max_out_degree) {
  if (!csr || !wedges || !max_out_degree || !(csr->flags & WETRIC_CSR_DEVICE)) {
    set_error(WETRIC_EINVAL, "wetric_wedge_total needs a device CSR");
    return WETRIC_EINVAL;
  }
  DeviceContext *ctx = nullptr;
  int st = get_context(device, &ctx);
  if (st == WETRIC_OK)
    st = wedge_total(ctx, ctx->stream, csr->row_ptr,
                     (csr->flags & WETRIC_CSR_OFFSETS32) != 0, csr->n, wedges,
                     max_out_degree);
  return finish(st);
}

int wetric_algorithmic_bytes(const wetric_csr *csr, int device,
                             uint64_t *bytes) {
  if (!csr || !bytes || !(csr->flags & WETRIC_CSR_DEVICE)) {
    set_error(WETRIC_EINVAL, "wetric_algorithmic_bytes needs a device CSR");
    return WETRIC_EINVAL;
  }
  DeviceContext *ctx = nullptr;
  int st = get_context(device, &ctx);
  if (st == WETRIC_OK)
    st = algorithmic_bytes(ctx, ctx->stream, csr->row_ptr,
                           (csr->flags & WETRIC_CSR_OFFSETS32) != 0,
                           csr->col_ind, csr->n, csr->m, bytes);
  return finish(st);
}

int wetric_orient_edges(const uint32_t *src, const uint32_t *dst,
                        uint64_t num_pairs, uint64_t n_hint, uint32_t flags,
                        int device, wetric_oriented *out, wetric_stats *stats) {
  if (!out || (num_pairs > 0 && (!src || !dst))) {
    set_error(WETRIC_EINVAL, "NULL argument");
    return WETRIC_EINVAL;
  }
  *out = nullptr;
  DeviceContext *ctx = nullptr;
  int st = get_context(device, &ctx);
  if (st != WETRIC_OK) return finish(st);
  cudaStream_t s = ctx->stream;
  wetric_stats ws = {};
  auto run = [&](wetric_oriented_s *h) -> int {
    const uint32_t *ds = src, *dd = dst;
    Scratch<uint32_t> bs, bd;
    if (!(flags & WETRIC_CSR_DEVICE)) {
      Timer tm;
      WETRIC_TRY(tm.start(s));
      WETRIC_TRY(bs.alloc(ctx, s, num_pairs));
      WETRIC_TRY(bd.alloc(ctx, s, num_pairs));
      if (num_pairs) {
        WETRIC_CUDA_TRY(cudaMemcpyAsync(bs.ptr, src, num_pairs * 4,
                                        cudaMemcpyHostToDevice, s));
        WETRIC_CUDA_TRY(cudaMemcpyAsync(bd.ptr, dst, num_pairs * 4,
                                        cudaMemcpyHostToDevice, s));
      }
      WETRIC_TRY(tm.stop(s, &ws.copy_ms));
      ds = bs.ptr;
      dd = bd.ptr;
    }
    Timer tp;
    WETRIC_TRY(tp.start(s));
    WETRIC_TRY(orient_pairs(ctx, s, ds, dd, num_pairs, n_hint, &h->csr));
    WETRIC_TRY(tp.stop(s, &ws.prep_ms));
    return WETRIC_OK;
  };
  wetric_oriented_s *h = new wetric_oriented_s();
  st = run(h);
  if (st != WETRIC_OK) {
    delete h;
    return finish(st);
  }
  ws.n = h->csr.n;
  ws.m = h->csr.m;
  if (stats) *stats = ws;
  *out = h;
  return finish(WETRIC_OK);
}

int wetric_oriented_csr(wetric_oriented h, wetric_csr *csr) {
  if (!h || !csr) {
    set_error(WETRIC_EINVAL, "NULL argument");
    return WETRIC_EINVAL;
  }
  csr->n = h->csr.n;
  csr->m = h->csr.m;
  csr->row_ptr = h->csr.row_ptr;
  csr->col_ind = h->csr.col_ind;
  csr->flags = WETRIC_CSR_ORIENTED | WETRIC_CSR_DEVICE;
  return finish(WETRIC_OK);
}

int wetric_oriented_download(wetric_oriented h, uint64_t *row_ptr,
                             uint32_t *col_ind) {
  if (!h || !row_ptr || (h->csr.m > 0 && !col_ind)) {
    set_error(WETRIC_EINVAL, "NULL argument");
    return WETRIC_EINVAL;
  }
  cudaStream_t s = h->csr.stream;
  auto run = [&]() -> int {
    WETRIC_CUDA_TRY(cudaSetDevice(h->csr.ctx->device));
    WETRIC_CUDA_TRY(cudaMemcpyAsync(row_ptr, h->csr.row_ptr,
                                    (h->csr.n + 1) * 8, cudaMemcpyDeviceToHost,
                                    s));
    if (h->csr.m)
      WETRIC_CUDA_TRY(cudaMemcpyAsync(col_ind, h->csr.col_ind, h->csr.m * 4,
                                      cudaMemcpyDeviceToHost, s));
    WETRIC_CUDA_TRY(cudaStreamSynchronize(s));
    return WETRIC_OK;
  };
  return finish(run());
}

void wetric_batch_opts_init(wetric_batch_opts *o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->spread = 5;
  o->bitmap_len = 8192;
  o->use_cuda_graph = 1;
}

// Spread for one graph of a batch when the caller asks for tuning: small
// graphs take short tiles so their few wedges still spread over many warps,
// large ones long tiles so warps stay on a row (the staged N+(w) is reused).
static uint32_t tuned_spread(uint64_t n, uint64_t W, const void *) {
  (void)n;
  if (W < (1ull << 16)) return 1;
  if (W < (1ull << 22)) return 2;
  if (W < (1ull << 28)) return 5;
  return 10;
}

int wetric_batch_create(const uint32_t *src, const uint32_t *dst,
                        const uint64_t *pair_off, const uint64_t *n,
                        uint32_t G, uint32_t flags, int device,
                        const wetric_batch_opts *opts, wetric_batch *out) {
  if (!out || !pair_off || !n || (G && pair_off[G] && (!src || !dst))) {
    set_error(WETRIC_EINVAL, "NULL argument");
    return WETRIC_EINVAL;
  }
  *out = nullptr;
  wetric_batch_opts o;
  if (opts) o = *opts; else wetric_batch_opts_init(&o);
  DeviceContext *ctx = nullptr;
  int st = get_context(device, &ctx);
  if (st != WETRIC_OK) return finish(st);
  BatchOptions bo;
  bo.spread = o.spread ? o.spread : 5;
  bo.spread_for = o.spread ? nullptr : tuned_spread;
  bo.bitmap_len = o.bitmap_len;
  bo.bitmap_cap_bytes = o.bitmap_cap_bytes ? o.bitmap_cap_bytes : (2ull << 30);
  bo.use_graph = o.use_cuda_graph != 0;
  bo.autotune = o.autotune != 0 && o.spread == 0;
  bo.pair_streams = o.no_pair_streams == 0;
  wetric_batch_s *h = new wetric_batch_s();
  st = batch_create(ctx, src, dst, pair_off, n, G,
                    (flags & WETRIC_CSR_DEVICE) != 0, bo, &h->batch);
  if (st != WETRIC_OK) {
    delete h;
    return finish(st);
  }
  *out = h;
  return finish(WETRIC_OK);
}

int wetric_batch_count(wetric_batch b, uint64_t *counts, wetric_stats *stats) {
  if (!b || !counts) {
    set_error(WETRIC_EINVAL, "NULL argument");
    return WETRIC_EINVAL;
  }
  double ms = 0;
  uint32_t launches = 0;
  const int st = batch_count(&b->batch, counts, &ms, &launches);
  if (st == WETRIC_OK && stats) {
    memset(stats, 0, sizeof(*stats));
    stats->exec_ms = ms;
    stats->count_ms = ms;
    stats->n = b->batch.vbase[b->batch.G];
    stats->m = b->batch.m_total;
    stats->wedges = b->batch.W + b->batch.pair_wedges;
    stats->wedges_counted = stats->wedges;
    stats->pair_rows = b->batch.Kp;
    stats->pair_wedges = b->batch.pair_wedges;
    stats->max_out_degree = b->batch.max_out_degree;
    stats->launches = launches;
    stats->spread = b->batch.opt.spread;
    stats->bitmap_len = b->batch.opt.bitmap_len;
  }
  return finish(st);
}

int wetric_batch_info(wetric_batch b, uint64_t *wedges, uint64_t *edges) {
  if (!b) {
    set_error(WETRIC_EINVAL, "NULL argument");
    return WETRIC_EINVAL;
  }
  const Batch &B = b->batch;
  if (wedges)
    for (uint32_t g = 0; g < B.G; ++g)
      wedges[g] = B.wbase[g + 1] - B.wbase[g] + (B.pair_w.empty() ? 0 : B.pair_w[g]);
  if (edges) {
    std::vector<uint64_t> e;
    const int st = batch_graph_edges(&b->batch, &e);
    if (st != WETRIC_OK) return finish(st);
    for (uint32_t g = 0; g < B.G; ++g) edges[g] = e[g];
  }
  return finish(WETRIC_OK);
}

int wetric_batch_spreads(wetric_batch b, uint32_t *spread) {
  if (!b || !spread) {
    set_error(WETRIC_EINVAL, "NULL argument");
    return WETRIC_EINVAL;
  }
  const Batch &B = b->batch;
  for (uint32_t g = 0; g < B.G; ++g) spread[g] = B.spread_of[g];
  return finish(WETRIC_OK);
}

void wetric_batch_free(wetric_batch b) {
  if (!b) return;
  cudaSetDevice(b->batch.ctx->device);
  cudaStream_t s = b->batch.stream;
  delete b;
  cudaStreamSynchronize(s);
}

void wetric_oriented_free(wetric_oriented h) {
  if (!h) return;
  if (h->csr.ctx) cudaSetDevice(h->csr.ctx->device);
  h->csr.release();
  if (h->csr.ctx) cudaStreamSynchronize(h->csr.stream);
  delete h;
}

}  // extern "C"
