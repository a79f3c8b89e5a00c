// batch.cuh -- many graphs counted in one persistent launch (see batch.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <vector>

#include "common.cuh"
#include "preprocess.cuh"

namespace wetric {

struct BatchOptions {
  uint32_t spread = 5;          // default s
  uint32_t bitmap_len = 8192;   // cap on every graph's bitmap length a_g
  uint64_t bitmap_cap_bytes = 1ull << 31;  // total bitmap memory cap
  bool use_graph = true;        // capture the count in a CUDA graph
  // Persistent count grid (SM count x occupancy) or one warp per tile: the
  // latter lets other streams' blocks in as the count's blocks finish.
  bool persistent = true;
  // Time candidate spreads per size/skew bucket (kept per device) instead
  // of taking spread_for / spread alone.
  bool autotune = false;
  // Optional tuner: spread for a graph with n vertices and W wedges.
  uint32_t (*spread_for)(uint64_t n, uint64_t W, const void *ctx) = nullptr;
  const void *tune_ctx = nullptr;
  // Pair streams for the short rows of every graph (32-bit offsets only):
  // counted by k_count_pairs beside the wedge check (pair_streams.cuh).
  bool pair_streams = true;
};

struct Batch {
  DeviceContext *ctx = nullptr;
  cudaStream_t stream = nullptr;
  uint32_t G = 0;
  BatchOptions opt;
  std::vector<uint64_t> n, vbase, wbase;
  uint64_t m_total = 0, W = 0, K = 0, max_out_degree = 0, bitmap_words = 0;
  DeviceCsr csr;
  bool off32 = false;
  Scratch<uint32_t> rp32;
  Scratch<uint64_t> act_wp, act_rb;
  Scratch<uint32_t> act_d, act_g;
  Scratch<uint32_t> bm;
  Scratch<uint64_t> bm_first, bm_S, bm_off, vbase_d;
  Scratch<uint32_t> ginfo;  // per-graph 32-byte records (BatchView::ginfo)
  Scratch<unsigned long long> counts, total;
  // Per-row hash sets (hash_buckets == 0 when they did not fit): bucket
  // prefix (build), per-row {first bucket, buckets} (lookups), buckets.
  Scratch<uint64_t> hoff;
  Scratch<uint2> hrows;
  Scratch<uint32_t> htab;
  uint64_t hash_buckets = 0;
  // One tile space over every graph: graph g's wedges are cut into tiles
  // of tile_size[g] = 256 * s_g wedges; tile_prefix[g] = first tile of g.
  std::vector<uint32_t> spread_of;
  uint64_t tiles = 0;
  Scratch<uint64_t> tile_prefix, wbase_d;
  Scratch<uint32_t> tile_size, tile_k;
  Scratch<unsigned long long> next_tile;
  uint64_t grid_max = 0;
  // Pair streams: Kp vertices (pv) with their graphs (pg) and the prefix
  // of their streamed columns (ps, Kp + 1 entries), in ptiles tiles of
  // ptile_cols columns (ptile_k: first vertex of each tile); pair_w[g]:
  // graph g's wedges counted by them (host).
  uint64_t Kp = 0, ptiles = 0, ptile_cols = 0, pair_wedges = 0;
  Scratch<uint32_t> pv, pg, ptile_k;
  Scratch<uint64_t> ps;
  std::vector<uint64_t> pair_w;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaStream_t graph_stream = nullptr;
  uint32_t graph_launches = 0;
  void release_all();
  ~Batch();
};

// Graph g owns pairs [pair_off[g], pair_off[g+1]) of src/dst with local ids
// below n[g] (pair_off and n are host arrays).
// Work runs on `stream` (0 = the context stream), which the batch keeps
// for its allocations.
int batch_create(DeviceContext *ctx, const uint32_t *src, const uint32_t *dst,
                 const uint64_t *pair_off, const uint64_t *n, uint32_t G,
                 bool on_device, const BatchOptions &opt, Batch *b,
                 cudaStream_t stream = nullptr);

// Oriented edges of every graph (host vector of G entries).
int batch_graph_edges(Batch *b, std::vector<uint64_t> *edges,
                      cudaStream_t stream = nullptr);

// Counts every graph (counts: host u64[G]); *ms = device time of the count.
// Runs on `stream` (0 = the batch's stream); synchronous.
int batch_count(Batch *b, uint64_t *counts, double *ms, uint32_t *launches,
                cudaStream_t stream = nullptr);

}  // namespace wetric
