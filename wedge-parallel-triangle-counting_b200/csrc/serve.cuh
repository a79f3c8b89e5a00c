// serve.cuh -- the resident serving engine: one persistent counting kernel
// that stays on the device and counts the tiles of every request the host
// publishes into its work queue, while other requests are still being
// preprocessed (serve.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "preprocess.cuh"

namespace wetric {

// Device buffers of one prepared request: its oriented CSR (u32 offsets)
// and everything the row-walk count reads -- active-vertex arrays, tile
// map, bitmap, 32-bit hash sets and 16-bit near sets (kernel 8's edge-check
// structures). Held until the engine retires the request.
struct ServePlan {
  DeviceCsr csr;  // from orientation (u64 offsets)
  Scratch<uint32_t> rp32;
  Scratch<uint64_t> act_wp, act_rb;
  Scratch<uint32_t> act_d, tile_k, bm, htab, ntab;
  Scratch<uint2> hrows, nrows;
  uint64_t n = 0, m = 0, W = 0, K = 0, tiles = 0, T = 0, bm_first = 0, S = 0;
  uint64_t max_out_degree = 0;
  uint32_t nfirst = 0, ncount = 0;
  uint64_t bytes = 0;  // device bytes held by the plan (approximate)
  // Dense core and shell of a large skewed request: counted by their own
  // kernels on the lane's stream beside the resident kernel (into core_acc,
  // done when core_done completes); the resident kernel's tiles cover the
  // wedges below the shell only.
  Scratch<uint32_t> core;
  Scratch<unsigned long long> core_acc;
  cudaEvent_t core_done = nullptr;
  uint64_t core_len = 0, shell_len = 0, core_wedges = 0;
  // Pair streams for the short rows (pair_streams.cuh): counted like the
  // core, on the lane's stream into core_acc before core_done.
  Scratch<uint32_t> pv, ptile_k;
  Scratch<uint64_t> ps;
  uint64_t pair_rows = 0, pair_wedges = 0;
  ~ServePlan() {
    if (core_done) cudaEventDestroy(core_done);
  }
};

// Builds every structure of plan->csr's count on `st` and waits for them:
// the work of count_oriented up to (not including) the count launch.
int serve_prepare(DeviceContext *ctx, cudaStream_t st, uint32_t spread,
                  uint32_t bitmap_len, ServePlan *plan);

struct ServeEngine;

struct ServeEngineOptions {
  uint32_t max_slots = 8192;      // requests per sequence space
  uint32_t max_items = 1u << 20;  // queue items per sequence space
  uint32_t idle_us = 2000;        // the kernel exits after this long idle
  uint32_t blocks_per_sm = 0;     // 0 = half the kernel's occupancy
};

int serve_engine_create(DeviceContext *ctx, const ServeEngineOptions &o,
                        ServeEngine **out);
void serve_engine_destroy(ServeEngine *e);

// Registers a prepared request: returns its slot and takes the plan, or
// WETRIC_EBUSY (the plan stays with the caller) when the sequence space is
// full (serve_recycle, then retry).
int serve_add(ServeEngine *e, std::unique_ptr<ServePlan> &plan, uint32_t *slot);
// Publishes the slot's tiles [t0, t1) as one queue item (WETRIC_EBUSY when
// the queue is full).
int serve_publish(ServeEngine *e, uint32_t slot, uint64_t t0, uint64_t t1);
// Launches the resident kernel when it is not running and published work
// is pending (memory of retired requests is freed first).
int serve_kick(ServeEngine *e);
// Completed slots since the last call: (slot, triangles). A slot with no
// tiles completes here too. Completed plans are retired.
int serve_poll(ServeEngine *e, std::vector<std::pair<uint32_t, uint64_t>> *done);
// Queue items the kernel has taken so far and items published.
void serve_queue_state(ServeEngine *e, uint64_t *taken, uint64_t *published);
// Lets the kernel drain and end, frees retired memory and starts a fresh
// sequence space (every registered slot must have completed).
int serve_recycle(ServeEngine *e);
// Device bytes held by retired (completed, not yet freed) requests, and
// the total of plan bytes freed so far (ServePlan::bytes, monotonic).
uint64_t serve_retired_bytes(ServeEngine *e);
uint64_t serve_freed_bytes(ServeEngine *e);
// Launches of the resident kernel so far and the last one's exit status
// (1 = stopped, 2 = gave up waiting on an empty queue).
void serve_launch_info(ServeEngine *e, uint64_t *launches, uint32_t *last_exit);
// Launches of the resident kernel that failed to start (and the
// cudaError_t of the last one).
uint64_t serve_launch_errors(ServeEngine *e, uint32_t *last_code = nullptr);
// Slots and items left in the current sequence space.
void serve_space_left(ServeEngine *e, uint32_t *slots, uint32_t *items);

// Runs the resident kernel once on an empty queue with a short idle limit
// and returns its exit status through *exit_code (2 = gave up waiting):
// the bounded wait, checked without a fault.
int serve_idle_probe(DeviceContext *ctx, uint32_t idle_us, uint32_t *exit_code,
                     double *ms);

}  // namespace wetric
