// batch.cu -- many graphs of uneven sizes counted in one persistent launch.
//
// The reference counts one graph per process run (tc.cu:896-913). Here a
// batch of G graphs is preprocessed once as a disjoint union (graph g owns
// ids [vbase[g], vbase[g+1]) and is ranked inside its own range, so its
// oriented CSR equals the one it gets alone), kept resident on the device,
// and counted by the row-walk kernel over the union's wedge space: every
// tile the persistent warps pull from the device work counter is a
// (graph, wedge-range) piece, and hits accumulate per graph. Each graph has
// its own bitmap over its last min(a, n_g) vertices and per-row hash sets
// for its longer rows below the bitmap; graph g's tiles hold 256 * s_g
// wedges, s_g from the autotuner's per-device table of size/skew buckets
// (or a size table); the count is captured once in a CUDA graph and
// replayed per count.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <numeric>
#include <vector>

#include "batch.cuh"
#include "count.cuh"
#include "count_kernels.cuh"
#include "pair_streams.cuh"
#include "preprocess.cuh"
#include "primitives.cuh"

namespace wetric {

namespace {

// The batch count is k_count_rows with long-row segments and per-row hash
// sets (skipped at run time when absent), at 5 blocks per SM.
constexpr int kBatchMinBlocks = 5;
// Resident hash sets: rows with d+ >= 16, three columns per bucket on average
// (about 11 bytes per hashed column).
constexpr uint32_t kBatchHashMinDegree = 16;
constexpr uint32_t kBatchHashKeysPerBucket = 3;

// Grid of a grid-stride element-wise kernel: at most 32 blocks per SM, so
// blocks stay short and a higher-priority stream's kernels get SMs soon.
unsigned grid_for(DeviceContext *ctx, uint64_t work, uint32_t block = 256) {
  const uint64_t cap = (uint64_t)ctx->sm_count * 32;
  uint64_t g = ceil_div(work, block);
  if (g > cap) g = cap;
  if (g == 0) g = 1;
  return (unsigned)g;
}

__device__ __forceinline__ uint32_t group_of(const uint64_t *__restrict__ base,
                                             uint32_t G, uint64_t x) {
  uint32_t lo = 0, len = G;
  while (len > 1) {
    const uint32_t h = len >> 1;
    if (base[lo + h] <= x) lo += h;
    len -= h;
  }
  return lo;
}

// Local pair ids -> union ids (graph found from the pair offsets); an id
// outside its graph's range raises *err.
__global__ void k_shift_pairs(uint32_t *__restrict__ src,
                              uint32_t *__restrict__ dst, uint64_t P,
                              const uint64_t *__restrict__ pair_off,
                              const uint64_t *__restrict__ vbase, uint32_t G,
                              uint32_t *err) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t g = group_of(pair_off, G, i);
    const uint64_t b = vbase[g], ng = vbase[g + 1] - b;
    const uint32_t s = src[i], d = dst[i];
    if ((uint64_t)s >= ng || (uint64_t)d >= ng) {
      atomicCAS(err, 0u, (uint32_t)kDevColumnRange);
      src[i] = dst[i] = (uint32_t)b;  // a self-loop: dropped downstream
    } else {
      src[i] = (uint32_t)(b + s);
      dst[i] = (uint32_t)(b + d);
    }
  }
}

__global__ void k_active_graph(const uint32_t *__restrict__ active, uint64_t n,
                               const uint64_t *__restrict__ pos,
                               const uint64_t *__restrict__ vbase, uint32_t G,
                               uint32_t *__restrict__ act_g) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x)
    if (active[v]) act_g[pos[v]] = group_of(vbase, G, v);
}

// wbase[g] = wedges before graph g = act_wp[pos[vbase[g]]].
__global__ void k_graph_wedge_base(const uint64_t *__restrict__ vbase,
                                   uint32_t G, const uint64_t *__restrict__ pos,
                                   const uint64_t *__restrict__ act_wp,
                                   uint64_t *__restrict__ wbase) {
  for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g <= G;
       g += (uint64_t)gridDim.x * blockDim.x)
    wbase[g] = act_wp[pos[vbase[g]]];
}

// One thread per union row: rows in the last a_g local ids of their graph
// set their bits in that graph's bitmap.
template <typename Off>
__global__ void k_batch_bitmap(const Off *__restrict__ rp,
                               const uint32_t *__restrict__ ci, uint64_t n,
                               const uint64_t *__restrict__ vbase, uint32_t G,
                               const uint64_t *__restrict__ bm_first,
                               const uint64_t *__restrict__ bm_S,
                               const uint64_t *__restrict__ bm_off,
                               uint32_t *__restrict__ bm) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t g = group_of(vbase, G, v);
    const uint64_t vb = vbase[g], ng = vbase[g + 1] - vb, vl = v - vb;
    const uint64_t Sg = bm_S[g];
    // Rows below the graph's first bitmap row carry no bits; the first row
    // n_g - min(n_g, a_g) equals the check threshold max(n_g, a_g) - a_g.
    if (Sg == 0 || vl < bm_first[g]) continue;
    const uint64_t base = Sg - (ng - vl) * (ng - vl - 1) / 2;
    const uint64_t e = (uint64_t)rp[v + 1];
    for (uint64_t j = (uint64_t)rp[v]; j < e; ++j) {
      const uint64_t w = ci[j];
      if (w <= v || w >= vb + ng) continue;
      const uint64_t idx = base + (w - vb) - vl - 1;
      if (idx < Sg) atomicOr(&bm[bm_off[g] + (idx >> 5)], 1u << (idx & 31));
    }
  }
}

// Hash-set buckets of every union row: rows of graph g below its bitmap
// (local id < bm_first[g]) with d+ >= kHashMinDegree.
template <typename Off>
__global__ void k_batch_hash_sizes(const Off *__restrict__ rp, uint64_t n,
                                   const uint64_t *__restrict__ vbase,
                                   uint32_t G,
                                   const uint64_t *__restrict__ bm_first,
                                   uint32_t *__restrict__ nb) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t g = group_of(vbase, G, v);
    nb[v] = v - vbase[g] < bm_first[g]
                ? hash_buckets_for((uint64_t)rp[v + 1] - (uint64_t)rp[v],
                                   kBatchHashMinDegree, kBatchHashKeysPerBucket)
                : 0u;
  }
}

// wedges of graph g counted by pair streams: atomics per pair vertex.
__global__ void k_pair_graph_wedges(const uint32_t *__restrict__ rp,
                                    const uint32_t *__restrict__ pv,
                                    const uint32_t *__restrict__ pg, uint64_t Kp,
                                    unsigned long long *__restrict__ w) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < Kp;
       k += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = pv[k];
    const uint64_t d = rp[v + 1] - rp[v];
    atomicAdd(w + pg[k], (unsigned long long)(d * (d - 1) / 2));
  }
}

// out[g] = row offset of graph g's first id (g <= G), so out[g+1] - out[g]
// is graph g's oriented edge count.
__global__ void k_first_offsets(const uint64_t *__restrict__ rp,
                                const uint64_t *__restrict__ vbase, uint32_t G,
                                uint64_t *__restrict__ out) {
  for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g <= G;
       g += (uint64_t)gridDim.x * blockDim.x)
    out[g] = rp[vbase[g]];
}

}  // namespace

int batch_graph_edges(Batch *b, std::vector<uint64_t> *edges, cudaStream_t stream) {
  cudaStream_t st = stream ? stream : b->stream;
  const uint32_t G = b->G;
  Scratch<uint64_t> first;
  WETRIC_TRY(first.alloc(b->ctx, st, G + 1));
  k_first_offsets<<<grid_for(b->ctx, G + 1), 256, 0, st>>>(b->csr.row_ptr, b->vbase_d.ptr,
                                                          G, first.ptr);
  WETRIC_LAUNCH_CHECK();
  std::vector<uint64_t> rpb(G + 1, 0);
  WETRIC_CUDA_TRY(cudaMemcpyAsync(rpb.data(), first.ptr, (G + 1) * 8,
                                  cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  edges->assign(G, 0);
  for (uint32_t g = 0; g < G; ++g) (*edges)[g] = rpb[g + 1] - rpb[g];
  return WETRIC_OK;
}

void Batch::release_all() {
  if (graph_exec) cudaGraphExecDestroy(graph_exec);
  if (graph) cudaGraphDestroy(graph);
  graph_exec = nullptr;
  graph = nullptr;
}

Batch::~Batch() { release_all(); }

// Sizes the per-graph bitmaps: a_g = min(a, n_g rounded up to 32), and no
// bitmap for graphs whose bitmap would push the total over the cap.
static void plan_bitmaps(const std::vector<uint64_t> &ng, uint32_t a,
                         uint64_t cap_words, std::vector<uint64_t> *first,
                         std::vector<uint64_t> *S, std::vector<uint64_t> *off,
                         uint64_t *total_words) {
  const size_t G = ng.size();
  first->assign(G, 0);
  S->assign(G, 0);
  off->assign(G, 0);
  uint64_t words = 0;
  for (size_t g = 0; g < G; ++g) {
    uint64_t ag = std::min<uint64_t>(a, (ng[g] + 31) / 32 * 32);
    uint64_t Sg = ag * (ag ? ag - 1 : 0) / 2;
    uint64_t wg = ceil_div(Sg, 32);
    if (ag < 2 || words + wg > cap_words) {
      ag = 0;
      Sg = 0;
      wg = 0;
    }
    (*first)[g] = ag ? (std::max<uint64_t>(ng[g], ag) - ag) : ng[g];
    (*S)[g] = Sg;
    (*off)[g] = words;
    words += wg;
  }
  *total_words = words;
}

static BatchView batch_view(const Batch *b) {
  BatchView bv;
  bv.G = b->G;
  bv.tile_prefix = b->tile_prefix.ptr;
  bv.tile_size = b->tile_size.ptr;
  bv.wbase = b->wbase_d.ptr;
  bv.act_g = b->act_g.ptr;
  bv.vbase = b->vbase_d.ptr;
  bv.bm_first = b->bm_first.ptr;
  bv.bm_S = b->bm_S.ptr;
  bv.bm_off = b->bm_off.ptr;
  bv.ginfo = b->ginfo.ptr;
  bv.counts = b->counts.ptr;
  return bv;
}

// Tile space for per-graph spreads sg (sg[g] == 0: graph g gets no tiles,
// which the autotuner uses to time one bucket alone).
static int build_tile_space(Batch *b, const std::vector<uint32_t> &sg,
                            cudaStream_t st) {
  const uint32_t G = b->G;
  b->spread_of = sg;
  std::vector<uint64_t> tprefix(G + 1, 0);
  std::vector<uint32_t> tsize(G);
  for (uint32_t g = 0; g < G; ++g) {
    const uint64_t Wg = b->wbase[g + 1] - b->wbase[g];
    tsize[g] = 256u * (sg[g] ? sg[g] : 1u);
    tprefix[g + 1] = tprefix[g] + (Wg && sg[g] ? ceil_div(Wg, tsize[g]) : 0);
  }
  b->tiles = tprefix[G];
  WETRIC_TRY(b->tile_prefix.alloc(b->ctx, st, G + 1));
  WETRIC_TRY(b->tile_size.alloc(b->ctx, st, G));
  WETRIC_TRY(b->tile_k.alloc(b->ctx, st, b->tiles + 1));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(b->tile_prefix.ptr, tprefix.data(), (G + 1) * 8,
                                  cudaMemcpyHostToDevice, st));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(b->tile_size.ptr, tsize.data(), G * 4,
                                  cudaMemcpyHostToDevice, st));
  if (b->tiles) {
    BatchView bv = batch_view(b);
    k_batch_tile_map<<<grid_for(b->ctx, b->tiles), 256, 0, st>>>(
        b->act_wp.ptr, b->K, b->tiles, bv, b->tile_k.ptr);
    WETRIC_LAUNCH_CHECK();
  }
  // host copies above read stack vectors: finish them before returning
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  return WETRIC_OK;
}

static int batch_enqueue(Batch *b, cudaStream_t st, uint32_t *launches);

// Size/skew bucket of a graph with W wedges and m oriented edges: wedges
// in factor-4 steps, wedges per edge in four classes (< 4, < 16, < 64,
// more), so graphs whose tiles behave alike share a spread.
static uint32_t tune_bucket(uint64_t W, uint64_t m) {
  uint32_t size = 0;
  while (size < 31 && (W >> (2 * (size + 1))) != 0) ++size;
  const uint64_t per_edge = m ? W / m : W;
  const uint32_t skew = per_edge < 4 ? 0 : per_edge < 16 ? 1 : per_edge < 64 ? 2 : 3;
  return size * 4 + skew;
}

// The autotuner: for every size/skew bucket of this batch that the device's
// table does not hold yet (and that has enough wedges to time), count the
// bucket's graphs alone with each candidate spread (tile = 256 * s wedges
// per warp) and keep the fastest; the table outlives the batch, so later
// batches on the device reuse it. The per-graph bitmaps (a_g = min(a, n_g))
// and the block (8 warps, the count kernel's register budget) are fixed.
static int autotune_spreads(Batch *b, std::vector<uint32_t> *sg, cudaStream_t st) {
  static const uint32_t kCandidates[] = {1, 2, 5, 10, 20};
  const uint32_t G = b->G;
  std::vector<uint64_t> edges;
  WETRIC_TRY(batch_graph_edges(b, &edges, st));
  std::vector<uint32_t> bucket(G);
  std::map<uint32_t, uint64_t> bucket_w;
  for (uint32_t g = 0; g < G; ++g) {
    const uint64_t Wg = b->wbase[g + 1] - b->wbase[g];
    bucket[g] = tune_bucket(Wg, edges[g]);
    bucket_w[bucket[g]] += Wg;
  }
  DeviceContext *ctx = b->ctx;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  WETRIC_CUDA_TRY(cudaEventCreate(&e0));
  WETRIC_CUDA_TRY(cudaEventCreate(&e1));
  int rc = WETRIC_OK;
  for (const auto &kv : bucket_w) {
    {
      std::lock_guard<std::mutex> lk(ctx->mu);
      if (ctx->spread_table.count(kv.first)) continue;
    }
    if (kv.second < (1ull << 20)) continue;  // too little work to time
    float best_ms = 0;
    uint32_t best_s = 0;
    for (uint32_t s : kCandidates) {
      std::vector<uint32_t> trial(G, 0);
      for (uint32_t g = 0; g < G; ++g)
        if (bucket[g] == kv.first) trial[g] = s;
      rc = build_tile_space(b, trial, st);
      if (rc != WETRIC_OK) break;
      uint32_t nl = 0;
      float ms = 0;
      for (int rep = 0; rep < 2 && rc == WETRIC_OK; ++rep) {  // warm, then time
        if (cudaEventRecord(e0, st) != cudaSuccess) rc = WETRIC_ECUDA;
        if (rc == WETRIC_OK) rc = batch_enqueue(b, st, &nl);
        if (rc == WETRIC_OK && (cudaEventRecord(e1, st) != cudaSuccess ||
                                cudaEventSynchronize(e1) != cudaSuccess ||
                                cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
          rc = WETRIC_ECUDA;
      }
      if (rc != WETRIC_OK) break;
      if (best_s == 0 || ms < best_ms) {
        best_ms = ms;
        best_s = s;
      }
    }
    if (rc != WETRIC_OK) break;
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->spread_table[kv.first] = best_s;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != WETRIC_OK) {
    if (rc == WETRIC_ECUDA) set_error(WETRIC_ECUDA, "batch autotuning failed");
    return rc;
  }
  std::lock_guard<std::mutex> lk(ctx->mu);
  for (uint32_t g = 0; g < G; ++g) {
    auto it = ctx->spread_table.find(bucket[g]);
    if (it != ctx->spread_table.end()) (*sg)[g] = it->second;
  }
  return WETRIC_OK;
}

int batch_create(DeviceContext *ctx, const uint32_t *src, const uint32_t *dst,
                 const uint64_t *pair_off, const uint64_t *n, uint32_t G,
                 bool on_device, const BatchOptions &opt, Batch *b,
                 cudaStream_t stream) {
  NvtxRange nvtx_("wetric batch create");
  cudaStream_t st = stream ? stream : ctx->stream;
  b->ctx = ctx;
  b->stream = st;
  b->G = G;
  b->opt = opt;
  if (G == 0) {
    set_error(WETRIC_EINVAL, "empty batch");
    return WETRIC_EINVAL;
  }
  if (opt.spread == 0 || opt.bitmap_len % 32 != 0) {
    set_error(WETRIC_EINVAL, "batch needs s > 0 and a %% 32 == 0");
    return WETRIC_EINVAL;
  }
  b->vbase.assign(G + 1, 0);
  b->n.assign(n, n + G);
  for (uint32_t g = 0; g < G; ++g) {
    if (n[g] == 0) {
      set_error(WETRIC_EINVAL, "graph %u has n = 0", g);
      return WETRIC_EINVAL;
    }
    b->vbase[g + 1] = b->vbase[g] + n[g];
    if (pair_off[g + 1] < pair_off[g]) {
      set_error(WETRIC_EINVAL, "pair offsets decrease at graph %u", g);
      return WETRIC_EINVAL;
    }
  }
  if (pair_off[0] != 0) {
    set_error(WETRIC_EINVAL, "pair offsets must start at 0");
    return WETRIC_EINVAL;
  }
  const uint64_t NT = b->vbase[G];
  if (NT >= (1ull << 32)) {
    set_error(WETRIC_ERANGE, "batch holds %llu vertices (>= 2^32); split it",
              (unsigned long long)NT);
    return WETRIC_ERANGE;
  }
  const uint64_t P = pair_off[G];

  // 1. Union pairs on the device, shifted into each graph's id range.
  Scratch<uint64_t> d_vbase, d_poff;
  WETRIC_TRY(d_vbase.alloc(ctx, st, G + 1));
  WETRIC_TRY(d_poff.alloc(ctx, st, G + 1));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(d_vbase.ptr, b->vbase.data(), (G + 1) * 8,
                                  cudaMemcpyHostToDevice, st));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(d_poff.ptr, pair_off, (G + 1) * 8,
                                  cudaMemcpyHostToDevice, st));
  {
    Scratch<uint32_t> us, ud, err;
    WETRIC_TRY(us.alloc(ctx, st, P));
    WETRIC_TRY(ud.alloc(ctx, st, P));
    WETRIC_TRY(err.alloc(ctx, st, 1));
    WETRIC_CUDA_TRY(cudaMemsetAsync(err.ptr, 0, 4, st));
    const cudaMemcpyKind kind =
        on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (P) {
      WETRIC_CUDA_TRY(cudaMemcpyAsync(us.ptr, src, P * 4, kind, st));
      WETRIC_CUDA_TRY(cudaMemcpyAsync(ud.ptr, dst, P * 4, kind, st));
      k_shift_pairs<<<grid_for(ctx, P), 256, 0, st>>>(us.ptr, ud.ptr, P,
                                                      d_poff.ptr, d_vbase.ptr,
                                                      G, err.ptr);
      WETRIC_LAUNCH_CHECK();
    }
    uint32_t herr = 0;
    WETRIC_CUDA_TRY(cudaMemcpyAsync(&herr, err.ptr, 4, cudaMemcpyDeviceToHost, st));
    WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
    if (herr) {
      set_error(WETRIC_EINVAL, "a pair id is not below its graph's n");
      return WETRIC_EINVAL;
    }
    // 2. One preprocessing pipeline over the union, ranked per graph.
    WETRIC_TRY(orient_pairs(ctx, st, us.ptr, ud.ptr, P, NT, &b->csr,
                            d_vbase.ptr, G));
  }
  const uint64_t m = b->csr.m;
  b->m_total = m;

  // 3. u32 offsets when they fit.
  b->off32 = m < (1ull << 32);
  if (b->off32) {
    WETRIC_TRY(b->rp32.alloc(ctx, st, NT + 1));
    WETRIC_TRY(narrow_offsets(ctx, st, b->csr.row_ptr, NT, b->rp32.ptr));
  }

  // 4. Active vertices of the union with their graph.
  Scratch<uint32_t> active, err;
  Scratch<uint64_t> pos;
  Scratch<unsigned long long> md;
  WETRIC_TRY(active.alloc(ctx, st, NT));
  WETRIC_TRY(pos.alloc(ctx, st, NT + 1));
  WETRIC_TRY(md.alloc(ctx, st, 1));
  WETRIC_TRY(err.alloc(ctx, st, 1));
  WETRIC_CUDA_TRY(cudaMemsetAsync(md.ptr, 0, 8, st));
  WETRIC_CUDA_TRY(cudaMemsetAsync(err.ptr, 0, 4, st));
  if (b->off32)
    k_vertex_wedges<uint32_t><<<grid_for(ctx, NT), 256, 0, st>>>(
        b->rp32.ptr, NT, m, active.ptr, md.ptr, err.ptr);
  else
    k_vertex_wedges<uint64_t><<<grid_for(ctx, NT), 256, 0, st>>>(
        b->csr.row_ptr, NT, m, active.ptr, md.ptr, err.ptr);
  WETRIC_LAUNCH_CHECK();
  // Pair streams: the short rows that take them leave the active set
  // (flags and stream lengths per vertex, put in vertex order below, so a
  // tile of them stays within a graph or two).
  const bool pairs = b->off32 && opt.pair_streams && m > 0;
  Scratch<uint32_t> is_pair, plen;
  Scratch<uint64_t> ppos;
  Scratch<unsigned long long> pw;
  if (pairs) {
    WETRIC_TRY(is_pair.alloc(ctx, st, NT));
    WETRIC_TRY(plen.alloc(ctx, st, NT));
    WETRIC_TRY(ppos.alloc(ctx, st, NT + 1));
    WETRIC_TRY(pw.alloc(ctx, st, 3));
    WETRIC_CUDA_TRY(cudaMemsetAsync(pw.ptr, 0, 24, st));
    k_pair_plan<true><<<grid_for(ctx, NT), 256, 0, st>>>(b->rp32.ptr, b->csr.col_ind, NT,
                                                         active.ptr, is_pair.ptr, plen.ptr,
                                                         pw.ptr);
    WETRIC_LAUNCH_CHECK();
    WETRIC_TRY((prim::exclusive_scan<uint32_t, uint64_t>(ctx, st, is_pair.ptr,
                                                         ppos.ptr, NT)));
  }
  WETRIC_TRY((prim::exclusive_scan<uint32_t, uint64_t>(ctx, st, active.ptr,
                                                       pos.ptr, NT)));
  uint64_t K = 0, Kp = 0;
  unsigned long long maxdeg = 0, Wp = 0;
  WETRIC_CUDA_TRY(cudaMemcpyAsync(&K, pos.ptr + NT, 8, cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(&maxdeg, md.ptr, 8, cudaMemcpyDeviceToHost, st));
  unsigned long long pacc[3] = {0, 0, 0};  // (unordered count), wedges, columns
  if (pairs) {
    WETRIC_CUDA_TRY(cudaMemcpyAsync(&Kp, ppos.ptr + NT, 8, cudaMemcpyDeviceToHost, st));
    WETRIC_CUDA_TRY(cudaMemcpyAsync(pacc, pw.ptr, 24, cudaMemcpyDeviceToHost, st));
  }
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  if (maxdeg >= (1ull << 30)) {
    set_error(WETRIC_ERANGE, "max out-degree %llu >= 2^30", maxdeg);
    return WETRIC_ERANGE;
  }
  b->K = K;
  b->max_out_degree = maxdeg;
  Wp = pacc[1];
  b->Kp = Kp;
  b->pair_wedges = Wp;
  b->pair_w.assign(G, 0);
  if (Kp) {
    // the pair vertices in order, their graphs and the prefix of their
    // streamed columns, then tiles over it
    WETRIC_TRY(b->pv.alloc(ctx, st, Kp));
    WETRIC_TRY(b->pg.alloc(ctx, st, Kp));
    WETRIC_TRY(b->ps.alloc(ctx, st, Kp + 1));
    Scratch<uint32_t> lens;
    WETRIC_TRY(lens.alloc(ctx, st, Kp));
    k_pair_compact<<<grid_for(ctx, NT), 256, 0, st>>>(is_pair.ptr, NT, ppos.ptr, plen.ptr,
                                                      b->pv.ptr, lens.ptr);
    WETRIC_LAUNCH_CHECK();
    k_active_graph<<<grid_for(ctx, NT), 256, 0, st>>>(is_pair.ptr, NT, ppos.ptr, d_vbase.ptr,
                                                      G, b->pg.ptr);
    WETRIC_LAUNCH_CHECK();
    WETRIC_TRY((prim::exclusive_scan<uint32_t, uint64_t>(ctx, st, lens.ptr, b->ps.ptr, Kp)));
    Scratch<unsigned long long> gw;
    WETRIC_TRY(gw.alloc(ctx, st, G));
    WETRIC_CUDA_TRY(cudaMemsetAsync(gw.ptr, 0, G * 8ull, st));
    k_pair_graph_wedges<<<grid_for(ctx, Kp), 256, 0, st>>>(b->rp32.ptr, b->pv.ptr, b->pg.ptr,
                                                           Kp, gw.ptr);
    WETRIC_LAUNCH_CHECK();
    uint64_t Rp = 0;
    WETRIC_CUDA_TRY(cudaMemcpyAsync(&Rp, b->ps.ptr + Kp, 8, cudaMemcpyDeviceToHost, st));
    WETRIC_CUDA_TRY(cudaMemcpyAsync(b->pair_w.data(), gw.ptr, G * 8ull,
                                    cudaMemcpyDeviceToHost, st));
    WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
    const uint64_t Tp = pair_tile_cols(Rp, ctx->sm_count);
    b->ptile_cols = Tp;
    b->ptiles = Rp ? ceil_div(Rp, Tp) : 0;
    if (b->ptiles) {
      WETRIC_TRY(b->ptile_k.alloc(ctx, st, b->ptiles + 1));
      k_tile_map<<<grid_for(ctx, b->ptiles + 1), 256, 0, st>>>(b->ps.ptr, Kp, 0, Rp, Tp,
                                                               b->ptiles, b->ptile_k.ptr);
      WETRIC_LAUNCH_CHECK();
    }
  }
  is_pair.release();
  plen.release();
  ppos.release();
  WETRIC_TRY(b->act_wp.alloc(ctx, st, K + 1));
  WETRIC_TRY(b->act_rb.alloc(ctx, st, K));
  WETRIC_TRY(b->act_d.alloc(ctx, st, K));
  WETRIC_TRY(b->act_g.alloc(ctx, st, K));
  if (K > 0) {
    if (b->off32)
      k_compact_active<uint32_t><<<grid_for(ctx, NT), 256, 0, st>>>(
          b->rp32.ptr, NT, active.ptr, pos.ptr, b->act_wp.ptr, b->act_rb.ptr,
          b->act_d.ptr);
    else
      k_compact_active<uint64_t><<<grid_for(ctx, NT), 256, 0, st>>>(
          b->csr.row_ptr, NT, active.ptr, pos.ptr, b->act_wp.ptr,
          b->act_rb.ptr, b->act_d.ptr);
    WETRIC_LAUNCH_CHECK();
    k_active_graph<<<grid_for(ctx, NT), 256, 0, st>>>(
        active.ptr, NT, pos.ptr, d_vbase.ptr, G, b->act_g.ptr);
    WETRIC_LAUNCH_CHECK();
  }
  WETRIC_TRY((prim::exclusive_scan<uint64_t, uint64_t>(ctx, st, b->act_wp.ptr,
                                                       b->act_wp.ptr, K)));
  Scratch<uint64_t> d_wbase;
  WETRIC_TRY(d_wbase.alloc(ctx, st, G + 1));
  k_graph_wedge_base<<<grid_for(ctx, G + 1), 256, 0, st>>>(
      d_vbase.ptr, G, pos.ptr, b->act_wp.ptr, d_wbase.ptr);
  WETRIC_LAUNCH_CHECK();
  b->wbase.assign(G + 1, 0);
  WETRIC_CUDA_TRY(cudaMemcpyAsync(b->wbase.data(), d_wbase.ptr, (G + 1) * 8,
                                  cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  b->W = b->wbase[G];
  active.release();
  pos.release();

  // 5. Per-graph bitmaps.
  std::vector<uint64_t> first, S, off;
  uint64_t words = 0;
  plan_bitmaps(b->n, opt.bitmap_len, opt.bitmap_cap_bytes / 4, &first, &S,
               &off, &words);
  WETRIC_TRY(b->bm.alloc(ctx, st, words ? words : 1));
  WETRIC_TRY(b->bm_first.alloc(ctx, st, G));
  WETRIC_TRY(b->bm_S.alloc(ctx, st, G));
  WETRIC_TRY(b->bm_off.alloc(ctx, st, G));
  WETRIC_TRY(b->vbase_d.alloc(ctx, st, G + 1));
  WETRIC_TRY(b->counts.alloc(ctx, st, G));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(b->bm_first.ptr, first.data(), G * 8,
                                  cudaMemcpyHostToDevice, st));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(b->bm_S.ptr, S.data(), G * 8,
                                  cudaMemcpyHostToDevice, st));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(b->bm_off.ptr, off.data(), G * 8,
                                  cudaMemcpyHostToDevice, st));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(b->vbase_d.ptr, b->vbase.data(), (G + 1) * 8,
                                  cudaMemcpyHostToDevice, st));
  // The count reads each graph's frame as one 32-byte record.
  std::vector<uint32_t> ginfo((size_t)G * 8, 0);
  for (uint32_t g = 0; g < G; ++g) {
    uint32_t *r = &ginfo[(size_t)g * 8];
    r[0] = (uint32_t)b->vbase[g];
    r[1] = (uint32_t)(b->vbase[g + 1] - b->vbase[g]);
    r[2] = (uint32_t)first[g];
    r[3] = (uint32_t)off[g];
    r[4] = (uint32_t)(off[g] >> 32);
    r[5] = (uint32_t)S[g];
    r[6] = (uint32_t)(S[g] >> 32);
  }
  WETRIC_TRY(b->ginfo.alloc(ctx, st, (size_t)G * 8));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(b->ginfo.ptr, ginfo.data(), (size_t)G * 32,
                                  cudaMemcpyHostToDevice, st));
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  b->bitmap_words = words;
  if (words) {
    WETRIC_CUDA_TRY(cudaMemsetAsync(b->bm.ptr, 0, words * 4, st));
    if (b->off32)
      k_batch_bitmap<uint32_t><<<grid_for(ctx, NT), 256, 0, st>>>(
          b->rp32.ptr, b->csr.col_ind, NT, d_vbase.ptr, G, b->bm_first.ptr,
          b->bm_S.ptr, b->bm_off.ptr, b->bm.ptr);
    else
      k_batch_bitmap<uint64_t><<<grid_for(ctx, NT), 256, 0, st>>>(
          b->csr.row_ptr, b->csr.col_ind, NT, d_vbase.ptr, G, b->bm_first.ptr,
          b->bm_S.ptr, b->bm_off.ptr, b->bm.ptr);
    WETRIC_LAUNCH_CHECK();
  }

  // 6. Per-row hash sets for the rows outside each graph's bitmap;
  //    left out (the count then searches) when they do not fit.
  {
    Scratch<uint32_t> nb;
    WETRIC_TRY(nb.alloc(ctx, st, NT));
    WETRIC_TRY(b->hoff.alloc(ctx, st, NT + 1));
    if (b->off32)
      k_batch_hash_sizes<uint32_t><<<grid_for(ctx, NT), 256, 0, st>>>(
          b->rp32.ptr, NT, d_vbase.ptr, G, b->bm_first.ptr, nb.ptr);
    else
      k_batch_hash_sizes<uint64_t><<<grid_for(ctx, NT), 256, 0, st>>>(
          b->csr.row_ptr, NT, d_vbase.ptr, G, b->bm_first.ptr, nb.ptr);
    WETRIC_LAUNCH_CHECK();
    WETRIC_TRY((prim::exclusive_scan<uint32_t, uint64_t>(ctx, st, nb.ptr,
                                                         b->hoff.ptr, NT)));
    uint64_t buckets = 0;
    WETRIC_CUDA_TRY(cudaMemcpyAsync(&buckets, b->hoff.ptr + NT, 8,
                                    cudaMemcpyDeviceToHost, st));
    WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
    nb.release();
    // The sets stay resident with the batch: take at most half of the
    // device memory that is free now.
    size_t free_b = 0, total_b = 0;
    WETRIC_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    const bool room = buckets * kHashBucket * 4 <= free_b / 2;
    if (buckets && room && buckets < (1ull << 32) &&
        b->htab.alloc(ctx, st, buckets * kHashBucket) == WETRIC_OK &&
        b->hrows.alloc(ctx, st, NT) == WETRIC_OK) {
      WETRIC_CUDA_TRY(cudaMemsetAsync(b->htab.ptr, 0xFF,
                                      buckets * kHashBucket * 4, st));
      if (b->off32)
        k_hash_build<uint32_t><<<grid_for(ctx, NT * 32), 256, 0, st>>>(
            b->rp32.ptr, b->csr.col_ind, NT, b->hoff.ptr, b->htab.ptr);
      else
        k_hash_build<uint64_t><<<grid_for(ctx, NT * 32), 256, 0, st>>>(
            b->csr.row_ptr, b->csr.col_ind, NT, b->hoff.ptr, b->htab.ptr);
      WETRIC_LAUNCH_CHECK();
      k_hash_rows<<<grid_for(ctx, NT), 256, 0, st>>>(b->hoff.ptr, NT, b->hrows.ptr);
      WETRIC_LAUNCH_CHECK();
      b->hash_buckets = buckets;
      b->hoff.release();  // the lookups read the per-row records
    } else {
      clear_error();
      b->hoff.release();
      b->htab.release();
    }
  }

  // 7. One tile space: graph g's wedges in tiles of 256 * s_g, s_g from
  //    the autotuner's per-device table (buckets of size and skew), the
  //    size table, or the batch's spread.
  WETRIC_TRY(b->wbase_d.alloc(ctx, st, G + 1));
  WETRIC_TRY(b->next_tile.alloc(ctx, st, 1));
  WETRIC_TRY(b->total.alloc(ctx, st, 1));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(b->wbase_d.ptr, b->wbase.data(), (G + 1) * 8,
                                  cudaMemcpyHostToDevice, st));
  int occ = 0;
  if (b->off32)
    WETRIC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &occ, k_count_rows<uint32_t, true, false, kBatchMinBlocks, true, true>, kWarpsPerBlock * 32, 0));
  else
    WETRIC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &occ, k_count_rows<uint64_t, true, false, kBatchMinBlocks, true, true>, kWarpsPerBlock * 32, 0));
  b->grid_max = (uint64_t)ctx->sm_count * (occ < 1 ? 1 : occ);

  std::vector<uint32_t> sg(G, opt.spread);
  for (uint32_t g = 0; g < G; ++g) {
    const uint64_t Wg = b->wbase[g + 1] - b->wbase[g];
    uint32_t s1 = opt.spread_for ? opt.spread_for(b->n[g], Wg, opt.tune_ctx) : opt.spread;
    sg[g] = s1 ? s1 : opt.spread;
  }
  if (opt.autotune) WETRIC_TRY(autotune_spreads(b, &sg, st));
  WETRIC_TRY(build_tile_space(b, sg, st));
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  return WETRIC_OK;
}

// The launches of one count: zero the outputs and the tile counter, then
// one persistent launch over the batch's whole tile space.
static int batch_enqueue(Batch *b, cudaStream_t st, uint32_t *launches) {
  WETRIC_CUDA_TRY(cudaMemsetAsync(b->counts.ptr, 0, b->G * 8ull, st));
  WETRIC_CUDA_TRY(cudaMemsetAsync(b->total.ptr, 0, 8, st));
  WETRIC_CUDA_TRY(cudaMemsetAsync(b->next_tile.ptr, 0, 8, st));
  *launches = 0;
  if (b->ptiles) {
    k_count_pairs<true><<<(unsigned)ceil_div(b->ptiles, kPairWarps), kPairWarps * 32, 0, st>>>(
        b->rp32.ptr, b->csr.col_ind, b->pv.ptr, b->ps.ptr, b->pg.ptr, b->Kp, b->ptile_k.ptr,
        b->ptiles, b->ptile_cols, nullptr, b->counts.ptr);
    WETRIC_LAUNCH_CHECK();
    *launches = 1;
  }
  if (!b->tiles) return WETRIC_OK;
  const BatchView bv = batch_view(b);
  const uint64_t NT = b->vbase[b->G];
  const uint64_t need = ceil_div(b->tiles, kWarpsPerBlock);
  const bool one_pass = !b->opt.persistent && need <= 0x7FFFFFFFull;
  uint64_t grid = one_pass ? need : b->grid_max;
  if (grid > need) grid = need;
  unsigned long long *counter = one_pass ? nullptr : b->next_tile.ptr;
  const HashView hv{b->hash_buckets ? b->hrows.ptr : nullptr, b->htab.ptr};
  if (b->off32)
    k_count_rows<uint32_t, true, false, kBatchMinBlocks, true, true><<<(unsigned)grid, kWarpsPerBlock * 32, 0, st>>>(
        b->rp32.ptr, b->csr.col_ind, NT, b->act_wp.ptr, b->act_rb.ptr,
        b->act_d.ptr, b->K, b->tile_k.ptr, b->tiles, 0, 0, 0, b->bm.ptr, 0, 0,
        counter, b->total.ptr, bv, hv);
  else
    k_count_rows<uint64_t, true, false, kBatchMinBlocks, true, true><<<(unsigned)grid, kWarpsPerBlock * 32, 0, st>>>(
        b->csr.row_ptr, b->csr.col_ind, NT, b->act_wp.ptr, b->act_rb.ptr,
        b->act_d.ptr, b->K, b->tile_k.ptr, b->tiles, 0, 0, 0, b->bm.ptr, 0, 0,
        counter, b->total.ptr, bv, hv);
  WETRIC_LAUNCH_CHECK();
  *launches += 1;
  return WETRIC_OK;
}

int batch_count(Batch *b, uint64_t *counts, double *ms, uint32_t *launches,
                cudaStream_t stream) {
  NvtxRange nvtx_("wetric batch count");
  cudaStream_t st = stream ? stream : b->stream;
  WETRIC_CUDA_TRY(cudaSetDevice(b->ctx->device));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  WETRIC_CUDA_TRY(cudaEventCreate(&e0));
  WETRIC_CUDA_TRY(cudaEventCreate(&e1));
  int rc = WETRIC_OK;
  uint32_t nl = 0;
  auto run = [&]() -> int {
    if (b->opt.use_graph && !b->graph_exec) {
      // Capture the count once; later calls replay it.
      b->graph_stream = st;
      WETRIC_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      const int r = batch_enqueue(b, st, &b->graph_launches);
      cudaGraph_t g = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(st, &g);
      if (r != WETRIC_OK) {
        if (g) cudaGraphDestroy(g);
        return r;
      }
      WETRIC_CUDA_TRY(ce);
      b->graph = g;
      WETRIC_CUDA_TRY(cudaGraphInstantiate(&b->graph_exec, g, 0));
    }
    WETRIC_CUDA_TRY(cudaEventRecord(e0, st));
    if (b->graph_exec) {
      WETRIC_CUDA_TRY(cudaGraphLaunch(b->graph_exec, st));
      nl = b->graph_launches;
    } else {
      WETRIC_TRY(batch_enqueue(b, st, &nl));
    }
    WETRIC_CUDA_TRY(cudaEventRecord(e1, st));
    WETRIC_CUDA_TRY(cudaMemcpyAsync(counts, b->counts.ptr, b->G * 8ull,
                                    cudaMemcpyDeviceToHost, st));
    WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
    float f = 0;
    WETRIC_CUDA_TRY(cudaEventElapsedTime(&f, e0, e1));
    *ms = f;
    return WETRIC_OK;
  };
  rc = run();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (launches) *launches = nl;
  return rc;
}

}  // namespace wetric
