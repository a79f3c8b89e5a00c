// count.cuh -- the wedge-parallel count on a device-resident oriented CSR.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace wetric {

struct CountArgs {
  uint64_t n = 0, m = 0;
  const void *row_ptr = nullptr;  // device, u64[n+1] or u32[n+1]
  bool offsets32 = false;
  const uint32_t *col_ind = nullptr;  // device, u32[m]
  uint32_t spread = 5;
  uint32_t bitmap_len = 0;
  uint32_t block = 0;  // 0 = default
  uint64_t wedge_begin = 0, wedge_end = 0;  // wedge_end == 0: to W
  bool validate = false;
  bool l2_persist = false;
  // Row-walk kernels (3-8): persistent grid (false: one warp per tile, so
  // other streams' blocks get SMs as the count's blocks end).
  bool persistent = true;
  // When set, col_ind is still being copied: the count waits for this event
  // (on its stream) before the first kernel that reads col_ind, so the
  // row-offset work overlaps the copy.
  cudaEvent_t ci_ready = nullptr;
  // Columns arriving in row chunks, highest rows first (host input): chunk
  // i holds rows [chunk_lo[i], chunk_lo[i - 1]) (chunk_lo[-1] = n, the
  // last chunk_lo 0) and is on the device once chunk_ready[i] has
  // completed. The count builds the bitmap rows and hash sets of a chunk
  // and counts the wedges of its vertices -- whose edge checks only read
  // rows above them -- while the chunks below are still copying. 0: no
  // chunks (ci_ready, when set, orders all columns). Not with validate.
  uint32_t col_chunks = 0;
  uint64_t chunk_lo[kMaxColChunks] = {};
  cudaEvent_t chunk_ready[kMaxColChunks] = {};
  // Called once the count's one host read-back has completed (and before
  // it waits on chunk_ready): the caller issues the column copies there,
  // so no copy is in flight while the read-back's device-to-host transfers
  // run (a read-back into pageable memory can otherwise queue behind them).
  int (*issue_copies)(void *) = nullptr;
  void *issue_ctx = nullptr;
  // Dense core (kernels 7 and 8): the top core_len vertices are counted by
  // row ANDs of a core bit matrix (k_core_count). 0 = sized from the row
  // offsets (at most 65536), kCoreOff = none, else that many (at most 65536).
  uint32_t core_len = 0;
  // Shell below the core (with the core matrix as the bitmap): 0 or
  // kCoreOff = none, else that many vertices.
  uint32_t shell_len = 0;
  // Pair streams for short rows (kernel 8, whole-graph counts with 32-bit
  // offsets whose columns are not copied in row chunks): vertices with d+ <= 64
  // whose pair streams cost less than their wedge checks are counted by
  // k_count_pairs instead (pair_streams.cuh). The count does not change.
  bool pair_streams = true;
  uint32_t kernel = 0;  // 0 = default (8), 1 = block-tile, 2 = warp-staged,
                        // 3 = row-walk with the shared-memory stage,
                        // 4 = row-walk, 5 = row-walk at 6 blocks/SM,
                        // 6 = 5 with per-row hash sets, 7 = 6 with
                        // long-row segments, 8 = 7 with 16-bit near
                        // hash sets
};

struct CountResult {
  uint64_t triangles = 0;
  uint64_t wedges = 0;          // W of the whole graph
  uint64_t wedges_counted = 0;  // wedges in the requested range
  uint64_t max_out_degree = 0;
  uint32_t block = 0, grid = 0, launches = 0;
  double exec_ms = 0.0;   // all device work of the count
  double count_ms = 0.0;  // the count kernels alone (wedge checks + core)
  double core_ms = 0.0;   // the core kernel alone
  uint64_t core_wedges = 0;  // wedges counted by the core kernel
  uint32_t core_len = 0;     // core vertices used (0: none)
  uint64_t shell_len = 0;    // shell vertices used (0: none)
  uint64_t shell_wedges = 0; // wedges counted by the shell kernel
  double shell_ms = 0.0;     // the shell kernel alone
  uint64_t pair_rows = 0;    // vertices counted by pair streams
  uint64_t pair_wedges = 0;  // their wedges
  double pair_ms = 0.0;      // the pair-stream kernel alone
};

constexpr uint32_t kCoreOff = 0xFFFFFFFFu;

// Counts the triangles closed by the wedges [wedge_begin, wedge_end) of an
// oriented CSR. Synchronous on `st` (it reads W back to size the launch).
int count_oriented(DeviceContext *ctx, cudaStream_t st, const CountArgs &a,
                   CountResult *r);

// W and the max out-degree of an oriented CSR.
int wedge_total(DeviceContext *ctx, cudaStream_t st, const void *row_ptr,
                bool offsets32, uint64_t n, uint64_t *W, uint64_t *maxdeg);

// Algorithmic bytes of the wedge-check count (see wetric.h).
int algorithmic_bytes(DeviceContext *ctx, cudaStream_t st, const void *row_ptr,
                      bool offsets32, const uint32_t *col_ind, uint64_t n,
                      uint64_t m, uint64_t *bytes);

// u64 -> u32 row offsets (m < 2^32).
int narrow_offsets(DeviceContext *ctx, cudaStream_t st, const uint64_t *rp64,
                   uint64_t n, uint32_t *rp32);
// u32 -> u64 row offsets.
int widen_offsets(DeviceContext *ctx, cudaStream_t st, const uint32_t *rp32,
                  uint64_t n, uint64_t *rp64);

}  // namespace wetric
