// count.cu -- wedge-parallel exact triangle count on an oriented CSR.
//
// The reference (tc.cu:315-441, tc.cu:173-293) builds its wedge prefix and
// bitmap on the host, copies them, and launches one 128-thread block per
// 128*s wedges; every thread binary-searches a 12-level constant-memory
// tree plus global memory for its first vertex, walks s wedges serially,
// and counts hits with a shared atomic per triangle.
//
// Here everything after the CSR copy runs on the device (kernels in
// count_kernels.cuh):
//   1. k_vertex_wedges   per-vertex "active" flag (d+ >= 2), row-offset
//                        checks, max out-degree; then k_pair_plan takes
//                        the short rows whose pair streams are cheaper out
//                        of the active set (pair_streams.cuh; counted by
//                        k_count_pairs before the wedge check)
//   2. scan + k_compact_active  active vertices only: act_wp (u64 wedge
//                        prefix), act_rb (row start), act_d (out-degree)
//   3. k_tile_map        the active vertex owning the first wedge of every
//                        tile; it replaces the constant-memory search tree
//                        (tc.cu:139-171, 306-313)
//   4. k_bitmap          the upper-triangular bit matrix over the last a
//                        vertices (tc.cu:329-346), with a ceiling word count
//   5. (kernels 6-8) k_hash_sizes + scan + k_hash_build: per-row hash
//                        sets for the rows outside the bitmap with d+ >= 16;
//                        kernel 8 builds the rows within 65536 ids of the
//                        end as 16-bit near sets (k_near_build)
//   6. the count kernel (opts.kernel):
//        1 k_count           block tiles, lane-per-wedge decode, tile prefix
//                            staged in shared memory
//        2 k_count_staged    warp tiles, 32-entry vertex window, N+(w)
//                            staged in shared memory
//        3/4/5 k_count_rows  warp tiles walked with warp-uniform (vertex,
//                            row, column) state; with/without the stage;
//                            5 = 6 blocks per SM
//        6                   k_count_rows at 6 blocks per SM with the hash
//                            sets for the edge check
//        7                   6 plus long-row segments: whole rounds inside
//                            one row of N+(v) check against a row-uniform
//                            bitmap row / hash set / search (segment_hits)
//        8 (default)         7 with the near sets: half the bytes per
//                            column for the most-probed hash rows
//      Every kernel counts in registers and adds one total per block.
//   Steps 1-3 and the set sizes read only the row offsets; one host
//   read-back then sizes the rest. With row chunks (host input, columns
//   still copying) the bitmap rows, sets and count of each chunk run as
//   the chunk arrives, highest rows first.
//
// Wedge order: vertex v (ascending), then (w_i, u_i) row-major over the
// strict upper triangle of N+(v) -- the order of tc.cu:194-244.
#include <cuda_runtime.h>
#include <stdint.h>

#include "count.cuh"
#include "count_kernels.cuh"
#include "pair_streams.cuh"
#include "primitives.cuh"

namespace wetric {

namespace {

constexpr int kSegsMinBlocks = 5;


// Grid of a grid-stride element-wise kernel: at most 32 blocks per SM, so
// blocks stay short and a higher-priority stream's kernels get SMs soon.
unsigned grid_for(DeviceContext *ctx, uint64_t work, uint32_t block = 256) {
  const uint64_t cap = (uint64_t)ctx->sm_count * 32;
  uint64_t g = ceil_div(work, block);
  if (g > cap) g = cap;
  if (g == 0) g = 1;
  return (unsigned)g;
}

struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  ~EventPair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
  int create() {
    WETRIC_CUDA_TRY(cudaEventCreate(&a));
    WETRIC_CUDA_TRY(cudaEventCreate(&b));
    return WETRIC_OK;
  }
};

// Host read-backs: one gather kernel collects the values into a device
// array and one copy brings them to pinned host memory. A copy into
// pageable memory (a stack variable) returns only when it is done, so one
// copy per value cost a round trip each while the device sat idle.
struct ReadSpan {
  const void *src;
  uint32_t count, bytes;  // elements of 4 or 8 bytes
};
constexpr uint32_t kReadSpans = 12;
constexpr uint32_t kReadWords = 128;
struct ReadPlan {
  ReadSpan s[kReadSpans];
  uint32_t n = 0, total = 0;
  // Returns the first word of the span in the gathered array.
  uint32_t add(const void *src, uint32_t count, uint32_t bytes) {
    s[n++] = ReadSpan{src, count, bytes};
    total += count;
    return total - count;
  }
};
__global__ void k_read_gather(ReadPlan p, uint64_t *__restrict__ out) {
  uint32_t base = 0;
  for (uint32_t i = 0; i < p.n; ++i) {
    const ReadSpan sp = p.s[i];
    for (uint32_t j = threadIdx.x; j < sp.count; j += blockDim.x)
      out[base + j] = sp.bytes == 4 ? (uint64_t)static_cast<const uint32_t *>(sp.src)[j]
                                    : static_cast<const uint64_t *>(sp.src)[j];
    base += sp.count;
  }
}
// Pinned words for the calling thread's read-backs (portable: any device),
// made on first use and freed when the thread ends; null if pinned memory
// cannot be had (the caller then reads into its own array).
uint64_t *readback_words() {
  struct Holder {
    uint64_t *p = nullptr;
    bool tried = false;
    ~Holder() {
      if (p) cudaFreeHost(p);
    }
  };
  thread_local Holder h;
  if (!h.tried) {
    h.tried = true;
    if (cudaHostAlloc(reinterpret_cast<void **>(&h.p), kReadWords * sizeof(uint64_t),
                      cudaHostAllocPortable) != cudaSuccess) {
      h.p = nullptr;
      cudaGetLastError();
    }
  }
  return h.p;
}
// Gathers plan's values on st, copies them to the host and waits (for
// `done`, recorded after the copy, when given); *words points at them
// afterwards (valid until the calling thread's next read).
int read_back(DeviceContext *ctx, cudaStream_t st, const ReadPlan &plan, uint64_t *local,
              const uint64_t **words, cudaEvent_t done = nullptr) {
  Scratch<uint64_t> dev;
  WETRIC_TRY(dev.alloc(ctx, st, plan.total));
  k_read_gather<<<1, 128, 0, st>>>(plan, dev.ptr);
  WETRIC_LAUNCH_CHECK();
  uint64_t *host = readback_words();
  if (!host) host = local;
  WETRIC_CUDA_TRY(cudaMemcpyAsync(host, dev.ptr, plan.total * sizeof(uint64_t),
                                  cudaMemcpyDeviceToHost, st));
  if (done) {
    WETRIC_CUDA_TRY(cudaEventRecord(done, st));
    WETRIC_CUDA_TRY(cudaEventSynchronize(done));
  } else {
    WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  }
  *words = host;
  return WETRIC_OK;
}

template <typename Off>
int count_impl(DeviceContext *ctx, cudaStream_t st, const CountArgs &a,
               CountResult *r) {
  NvtxRange nvtx_("wetric count");
  const Off *rp = static_cast<const Off *>(a.row_ptr);
  const uint64_t n = a.n, m = a.m;
  *r = CountResult();
  // Row chunks must cover the rows top down (and exclude validation, which
  // reads every column before the chunks arrive).
  const uint32_t C_in = a.col_chunks;
  if (C_in > kMaxColChunks || (C_in && a.validate)) {
    set_error(WETRIC_EINVAL, "bad column chunks");
    return WETRIC_EINVAL;
  }
  for (uint32_t i = 0; i < C_in; ++i) {
    const uint64_t hi = i ? a.chunk_lo[i - 1] : n;
    if (a.chunk_lo[i] >= hi || (i + 1 == C_in && a.chunk_lo[i] != 0)) {
      set_error(WETRIC_EINVAL, "column chunks must cover the rows top down");
      return WETRIC_EINVAL;
    }
  }
  EventPair ev_all;
  WETRIC_TRY(ev_all.create());
  WETRIC_CUDA_TRY(cudaEventRecord(ev_all.a, st));
  uint32_t launches = 0;

  Scratch<uint32_t> small;  // [0] err
  // [0] max degree, [1] count, [2..4] pair vertices, their wedges, their
  // streamed columns
  Scratch<unsigned long long> acc;
  WETRIC_TRY(small.alloc(ctx, st, 4));
  WETRIC_TRY(acc.alloc(ctx, st, 5));
  WETRIC_CUDA_TRY(cudaMemsetAsync(small.ptr, 0, 4 * sizeof(uint32_t), st));
  WETRIC_CUDA_TRY(
      cudaMemsetAsync(acc.ptr, 0, 5 * sizeof(unsigned long long), st));
  if (n == 0) {
    WETRIC_CUDA_TRY(cudaEventRecord(ev_all.b, st));
    WETRIC_CUDA_TRY(cudaEventSynchronize(ev_all.b));
    return WETRIC_OK;
  }

  Scratch<uint32_t> active;
  Scratch<uint64_t> pos;
  WETRIC_TRY(active.alloc(ctx, st, n));
  WETRIC_TRY(pos.alloc(ctx, st, n + 1));
  k_vertex_wedges<Off><<<grid_for(ctx, n), 256, 0, st>>>(rp, n, m, active.ptr,
                                                         acc.ptr, small.ptr);
  WETRIC_LAUNCH_CHECK();
  ++launches;
  if (a.validate && m > 0) {
    if (a.ci_ready) WETRIC_CUDA_TRY(cudaStreamWaitEvent(st, a.ci_ready, 0));
    k_validate<Off><<<grid_for(ctx, n * 32), 256, 0, st>>>(rp, a.col_ind, n, m,
                                                           small.ptr);
    WETRIC_LAUNCH_CHECK();
    ++launches;
  }
  // Pair streams (short rows): whole-graph counts whose columns are on the
  // device or already being copied whole, 32-bit offsets, kernel 8, at
  // least kPairMinColumns columns (below that the plan's launches cost more
  // than it saves). The vertices that take them leave the active set, so
  // the wedge check, the core and the shell never see them. Not with
  // validation: the plan reads columns before the count's read-back has
  // seen the validation's verdict.
  const uint32_t kid0 = a.kernel == 0 ? 8u : a.kernel;
  const bool pairs_on = a.pair_streams && sizeof(Off) == 4 && kid0 == 8 && C_in == 0 &&
                        !a.issue_copies && !a.validate && a.wedge_begin == 0 &&
                        a.wedge_end == 0 && m >= kPairMinColumns;
  Scratch<uint32_t> pv, pl;
  Scratch<uint64_t> ps;
  if (pairs_on) {
    WETRIC_TRY(pv.alloc(ctx, st, n));
    WETRIC_TRY(pl.alloc(ctx, st, n));
    // the plan reads columns: after their copy (already issued) when the
    // input came from the host
    if (a.ci_ready) WETRIC_CUDA_TRY(cudaStreamWaitEvent(st, a.ci_ready, 0));
    k_pair_plan<<<grid_for(ctx, n), 256, 0, st>>>(reinterpret_cast<const uint32_t *>(rp),
                                                  a.col_ind, n, active.ptr, pv.ptr, pl.ptr,
                                                  acc.ptr + 2);
    WETRIC_LAUNCH_CHECK();
    ++launches;
  }

  WETRIC_TRY((prim::exclusive_scan<uint32_t, uint64_t>(ctx, st, active.ptr,
                                                       pos.ptr, n)));
  launches += 3;

  // Active-vertex arrays sized for all n vertices, so nothing waits for K:
  // entries past K stay zero and leave the prefix at W (act_wp[n] == W).
  const uint32_t kid = a.kernel == 0 ? 8u : a.kernel;
  Scratch<uint64_t> act_wp, act_rb;
  Scratch<uint32_t> act_d;
  WETRIC_TRY(act_wp.alloc(ctx, st, n + 1));
  WETRIC_TRY(act_rb.alloc(ctx, st, n));
  WETRIC_TRY(act_d.alloc(ctx, st, n));
  WETRIC_CUDA_TRY(cudaMemsetAsync(act_wp.ptr, 0, (n + 1) * sizeof(uint64_t), st));
  k_compact_active<Off><<<grid_for(ctx, n), 256, 0, st>>>(
      rp, n, active.ptr, pos.ptr, act_wp.ptr, act_rb.ptr, act_d.ptr);
  WETRIC_LAUNCH_CHECK();
  ++launches;
  WETRIC_TRY((prim::exclusive_scan<uint64_t, uint64_t>(ctx, st, act_wp.ptr,
                                                       act_wp.ptr, n)));
  launches += 3;

  // Bucket counts of the per-row hash sets (kernels 6-8) from the row
  // offsets alone, so they come back with the same read-back.
  const bool staged_kernel = a.kernel != kKernelBlockTile;
  const uint64_t alen = a.bitmap_len;
  const uint64_t bm_first = (n > alen ? n : alen) - alen;  // tc.cu:262
  const bool want_hash = staged_kernel && (kid == 6 || kid == 7 || kid == 8);
  // Kernel 8: the hash rows within kNearSpan of the end, [nfirst,
  // bm_first), get 16-bit near sets instead.
  const uint64_t nfirst = (n > kNearSpan ? n : kNearSpan) - kNearSpan;
  const uint64_t ncount = kid == 8 && nfirst < bm_first ? bm_first - nfirst : 0;
  Scratch<uint64_t> hoff, noff;
  if (want_hash) {
    Scratch<uint32_t> nb;
    WETRIC_TRY(nb.alloc(ctx, st, n));
    WETRIC_TRY(hoff.alloc(ctx, st, n + 1));
    k_hash_sizes<Off><<<grid_for(ctx, n), 256, 0, st>>>(
        rp, n, ncount ? nfirst : bm_first, kHashMinDegree, kHashKeysPerBucket,
        nb.ptr);
    WETRIC_LAUNCH_CHECK();
    WETRIC_TRY((prim::exclusive_scan<uint32_t, uint64_t>(ctx, st, nb.ptr,
                                                         hoff.ptr, n)));
    launches += 4;
    if (ncount) {
      WETRIC_TRY(noff.alloc(ctx, st, ncount + 1));
      k_hash_sizes<Off><<<grid_for(ctx, ncount), 256, 0, st>>>(
          rp + nfirst, ncount, ncount, kHashMinDegree, kNearKeysPerBucket,
          nb.ptr);
      WETRIC_LAUNCH_CHECK();
      WETRIC_TRY((prim::exclusive_scan<uint32_t, uint64_t>(ctx, st, nb.ptr,
                                                           noff.ptr, ncount)));
      launches += 4;
    }
  }

  // Dense core (kernels 7 and 8): the candidate sizes' wedges and row-AND
  // words (row offsets only), and the first core wedge of each candidate,
  // so the one read-back below sizes the core too.
  const bool core_kernel = staged_kernel && (kid == 7 || kid == 8) &&
                           a.core_len != kCoreOff && n >= 64;
  Scratch<unsigned long long> cplan;
  Scratch<uint64_t> cstart;
  CoreStarts cs{};
  if (core_kernel) {
    // For each candidate core, its first vertex and the first vertex of the
    // shell below it (shell_len vertices; 0 or kCoreOff = no shell).
    auto push = [&](uint64_t h) {
      const uint64_t v0 = n - (n < h ? n : h);
      const uint64_t sh = a.shell_len == kCoreOff ? 0 : a.shell_len;
      cs.v0[cs.c++] = v0;
      cs.v0[cs.c++] = v0 > sh ? v0 - sh : 0;
    };
    if (a.core_len == 0) {
      WETRIC_TRY(cplan.alloc(ctx, st, 2 * kCoreNumCandidates));
      WETRIC_CUDA_TRY(cudaMemsetAsync(
          cplan.ptr, 0, 2 * kCoreNumCandidates * sizeof(unsigned long long), st));
      const uint64_t top = n < core_candidate(0) ? n : core_candidate(0);
      k_core_plan<Off><<<grid_for(ctx, top), 256, 0, st>>>(rp, n, cplan.ptr);
      WETRIC_LAUNCH_CHECK();
      ++launches;
      for (uint32_t c = 0; c < kCoreNumCandidates; ++c) push(core_candidate(c));
    } else {
      push(a.core_len < kCoreMaxLen ? a.core_len : kCoreMaxLen);
    }
    WETRIC_TRY(cstart.alloc(ctx, st, 2 * (2 * kCoreNumCandidates + 2)));
    k_core_prefix<<<1, 32, 0, st>>>(act_wp.ptr, pos.ptr, cs, cstart.ptr);
    WETRIC_LAUNCH_CHECK();
    ++launches;
  }

  // Row chunks (host input): the wedge prefix at each chunk's first row.
  Scratch<uint64_t> cpre;
  uint64_t chunk_w[kMaxColChunks] = {};
  if (C_in) {
    ChunkRows cr{};
    for (uint32_t i = 0; i < C_in; ++i) cr.v[i] = a.chunk_lo[i];
    cr.c = C_in;
    WETRIC_TRY(cpre.alloc(ctx, st, kMaxColChunks));
    k_chunk_prefix<<<1, 32, 0, st>>>(act_wp.ptr, pos.ptr, cr, cpre.ptr);
    WETRIC_LAUNCH_CHECK();
    ++launches;
  }

  // One read-back: K, max out-degree, the row check, W, the buckets, the
  // chunks' wedge offsets, the pair-stream totals and the core plan.
  uint64_t K = 0, W = 0, buckets = 0, nbuckets = 0;
  unsigned long long maxdeg = 0;
  uint32_t err = 0;
  unsigned long long pacc[3] = {0, 0, 0};  // pair vertices, wedges, columns
  unsigned long long plan[2 * kCoreNumCandidates] = {};
  uint64_t starts[2 * (2 * kCoreNumCandidates + 2)] = {};
  {
    ReadPlan rd;
    const uint32_t iK = rd.add(pos.ptr + n, 1, 8), iD = rd.add(acc.ptr, 1, 8),
                   iE = rd.add(small.ptr, 1, 4), iW = rd.add(act_wp.ptr + n, 1, 8);
    const uint32_t iB = want_hash ? rd.add(hoff.ptr + n, 1, 8) : 0;
    const uint32_t iN = ncount ? rd.add(noff.ptr + ncount, 1, 8) : 0;
    const uint32_t iC = C_in ? rd.add(cpre.ptr, C_in, 8) : 0;
    const uint32_t iP = pairs_on ? rd.add(acc.ptr + 2, 3, 8) : 0;
    const uint32_t iL = cplan.ptr ? rd.add(cplan.ptr, 2 * kCoreNumCandidates, 8) : 0;
    const uint32_t iS = cstart.ptr ? rd.add(cstart.ptr, 2 * cs.c, 8) : 0;
    uint64_t local[kReadWords];
    const uint64_t *w = nullptr;
    WETRIC_TRY(read_back(ctx, st, rd, local, &w));
    K = w[iK];
    maxdeg = w[iD];
    err = (uint32_t)w[iE];
    W = w[iW];
    if (want_hash) buckets = w[iB];
    if (ncount) nbuckets = w[iN];
    for (uint32_t i = 0; i < C_in; ++i) chunk_w[i] = w[iC + i];
    if (pairs_on)
      for (uint32_t i = 0; i < 3; ++i) pacc[i] = w[iP + i];
    if (cplan.ptr)
      for (uint32_t i = 0; i < 2 * kCoreNumCandidates; ++i) plan[i] = w[iL + i];
    if (cstart.ptr)
      for (uint32_t i = 0; i < 2 * cs.c; ++i) starts[i] = w[iS + i];
  }
  if (err != kDevOk) {
    set_error(WETRIC_EINVAL, "oriented CSR check failed (device code %u)", err);
    return WETRIC_EINVAL;
  }
  r->max_out_degree = maxdeg;
  if (maxdeg >= kMaxOutDegree) {
    set_error(WETRIC_ERANGE, "max out-degree %llu >= 2^30", maxdeg);
    return WETRIC_ERANGE;
  }
  if (a.issue_copies) WETRIC_TRY(a.issue_copies(a.issue_ctx));
  active.release();
  pos.release();
  const uint64_t Kp = pacc[0], Wp = pacc[1], Rp = pacc[2];
  r->wedges = W + Wp;
  r->pair_rows = Kp;
  r->pair_wedges = Wp;

  // The core: the eligible candidate of least estimated time (core_pick),
  // or the caller's length.
  uint64_t core_h = 0, core_v0 = n, core_K = 0, core_W = W;
  uint64_t shell_v1 = n, shell_K = 0, shell_W = W;
  if (core_kernel) {
    int pick = -1;
    if (a.core_len == 0) {
      pick = core_pick(plan);
    } else {
      pick = 0;
    }
    if (pick >= 0) {
      core_v0 = cs.v0[2 * pick];
      core_h = n - core_v0;
      core_K = starts[4 * pick];
      core_W = starts[4 * pick + 1];
      shell_v1 = cs.v0[2 * pick + 1];
      shell_K = starts[4 * pick + 2];
      shell_W = starts[4 * pick + 3];
    }
    if (core_h < 32) {  // too small to pay for its launches
      core_h = 0;
      core_v0 = n;
      core_W = W;
    }
  }
  // The shell needs the core matrix as the bitmap (the core covers the
  // bitmap's rows), so the checks of its non-AND pairs find every row.
  if (!core_h || core_h < a.bitmap_len || shell_v1 >= core_v0) {
    shell_v1 = core_v0;
    shell_K = core_K;
    shell_W = core_W;
  }
  r->core_len = (uint32_t)core_h;
  r->shell_len = core_v0 - shell_v1;

  const uint64_t wb = a.wedge_begin < W ? a.wedge_begin : W;
  const uint64_t we = (a.wedge_end == 0 || a.wedge_end > W) ? W : a.wedge_end;
  if (we <= wb && !Rp) {
    WETRIC_CUDA_TRY(cudaEventRecord(ev_all.b, st));
    WETRIC_CUDA_TRY(cudaEventSynchronize(ev_all.b));
    float ms = 0;
    WETRIC_CUDA_TRY(cudaEventElapsedTime(&ms, ev_all.a, ev_all.b));
    r->exec_ms = ms;
    r->launches = launches;
    return WETRIC_OK;
  }
  r->wedges_counted = (we > wb ? we - wb : 0) + Wp;

  // Chunks, highest rows first: rows [lo, hi), wedges [wlo, whi) of their
  // vertices (wedge order is vertex order), ready after `ready`. Without
  // row chunks, one chunk of all rows behind ci_ready.
  struct Chunk {
    uint64_t lo, hi, wlo, whi;
    cudaEvent_t ready;
    uint64_t tiles, toff;
  };
  Chunk ch[kMaxColChunks];
  uint64_t core_lo[kMaxColChunks] = {}, core_hi[kMaxColChunks] = {};
  const uint32_t C = C_in ? C_in : 1u;
  for (uint32_t i = 0; i < C; ++i) {
    ch[i].lo = C_in ? a.chunk_lo[i] : 0;
    ch[i].hi = i ? ch[i - 1].lo : n;
    ch[i].wlo = C_in ? chunk_w[i] : 0;
    ch[i].whi = i ? ch[i - 1].wlo : W;
    ch[i].ready = C_in ? a.chunk_ready[i] : a.ci_ready;
  }
  // Each chunk's share for the core (wedges [core_W, W)), the shell
  // ([shell_W, core_W)) and the wedge-check kernel (below shell_W), within
  // [wb, we).
  uint64_t shell_lo[kMaxColChunks] = {}, shell_hi[kMaxColChunks] = {};
  for (uint32_t i = 0; i < C; ++i) {
    const uint64_t lo0 = ch[i].wlo > wb ? ch[i].wlo : wb;
    const uint64_t hi0 = ch[i].whi < we ? ch[i].whi : we;
    core_lo[i] = lo0 > core_W ? lo0 : core_W;
    core_hi[i] = core_h && hi0 > core_lo[i] ? hi0 : core_lo[i];
    shell_lo[i] = lo0 > shell_W ? lo0 : shell_W;
    const uint64_t sh = hi0 < core_W ? hi0 : core_W;
    shell_hi[i] = sh > shell_lo[i] ? sh : shell_lo[i];
    if (core_h && ch[i].whi > shell_W) ch[i].whi = ch[i].wlo > shell_W ? ch[i].wlo : shell_W;
  }

  // Launch shape. Block-tile kernel: block threads, s wedges per thread
  // per tile, T + 1 staged prefix entries per block. Warp-staged kernel:
  // tiles of T = 256 * s wedges taken whole by one warp.
  uint32_t B = staged_kernel ? kWarpsPerBlock * 32
                             : (a.block ? a.block : kDefaultBlock);
  const uint32_t s = a.spread;
  const size_t smem_cap = 200 * 1024;
  while (!staged_kernel && B > 32 &&
         ((uint64_t)B * s + 1) * sizeof(uint64_t) > smem_cap)
    B >>= 1;
  if (!staged_kernel && ((uint64_t)B * s + 1) * sizeof(uint64_t) > smem_cap) {
    set_error(WETRIC_ERANGE, "spread %u too large", s);
    return WETRIC_ERANGE;
  }
  uint64_t T = (uint64_t)(staged_kernel ? 256 : B) * s;
  if (staged_kernel) {
    // Small wedge counts: shrink the warp tile (in whole rounds of 32
    // wedges) until there are about two tiles per warp slot of the device,
    // so a small graph still spreads over every SM instead of a few warps
    // walking long tiles.
    const uint64_t min_tiles = 2ull * (uint64_t)ctx->sm_count * 64;
    if (ceil_div(we - wb, T) < min_tiles) {
      const uint64_t t = ceil_div(ceil_div(we - wb, min_tiles), 32) * 32;
      T = t < T ? (t < 32 ? 32 : t) : T;
    }
  }
  // Each chunk's part of [wb, we) gets its own tiles and tile map entries.
  uint64_t tile_entries = 0;
  for (uint32_t i = 0; i < C; ++i) {
    const uint64_t cb = ch[i].wlo > wb ? ch[i].wlo : wb;
    const uint64_t ce = ch[i].whi < we ? ch[i].whi : we;
    ch[i].wlo = cb;
    ch[i].whi = ce > cb ? ce : cb;
    ch[i].tiles = ce > cb ? ceil_div(ce - cb, T) : 0;
    ch[i].toff = tile_entries;
    tile_entries += ch[i].tiles + 1;
    if (ch[i].tiles >= (1ull << 40)) {
      set_error(WETRIC_ERANGE, "too many tiles; raise the spread");
      return WETRIC_ERANGE;
    }
  }
  const size_t smem = staged_kernel ? 0 : (T + 1) * sizeof(uint64_t);

  Scratch<uint32_t> tile_k;
  WETRIC_TRY(tile_k.alloc(ctx, st, tile_entries));
  for (uint32_t i = 0; i < C; ++i) {
    if (!ch[i].tiles) continue;
    k_tile_map<<<grid_for(ctx, ch[i].tiles + 1), 256, 0, st>>>(
        act_wp.ptr, K, ch[i].wlo, ch[i].whi, T, ch[i].tiles,
        tile_k.ptr + ch[i].toff);
    WETRIC_LAUNCH_CHECK();
    ++launches;
  }

  // Bitmap over the last a vertices (tc.cu:329-346). S = a(a-1)/2 bits,
  // rounded up to whole words (the reference's S/32 drops up to 16 bits
  // when a % 64 == 32). Its rows are written chunk by chunk below.
  // When the dense core covers the bitmap's rows, the core matrix serves
  // as the count's bitmap (its rows are the same bits, word-aligned) and
  // the packed bitmap is not built.
  const bool aligned = core_h && core_h >= alen;
  const uint64_t S = alen * (alen ? alen - 1 : 0) / 2;
  const uint64_t words = aligned ? 0 : ceil_div(S, 32);
  const uint64_t first_row = n - (n < alen ? n : alen);
  Scratch<uint32_t> bm;
  WETRIC_TRY(bm.alloc(ctx, st, words ? words : 1));
  if (words)
    WETRIC_CUDA_TRY(cudaMemsetAsync(bm.ptr, 0, words * sizeof(uint32_t), st));

  // Optional L2 residency for the bitmap (opts.l2_persist): set aside L2
  // lines for persisting accesses in this process's context, up to the
  // device maximum, and mark the bitmap as one access-policy window on the
  // stream; both are undone after the count.
  cudaAccessPolicyWindow window = {};
  bool window_set = false;
  if (a.l2_persist && words && ctx->window_max > 0 && ctx->persist_max > 0) {
    size_t bytes = words * sizeof(uint32_t);
    if (bytes > ctx->window_max) bytes = ctx->window_max;
    size_t setaside = bytes < ctx->persist_max ? bytes : ctx->persist_max;
    WETRIC_CUDA_TRY(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, setaside));
    window.base_ptr = bm.ptr;
    window.num_bytes = bytes;
    window.hitRatio = (float)setaside / (float)bytes;
    window.hitProp = cudaAccessPropertyPersisting;
    window.missProp = cudaAccessPropertyStreaming;
    cudaStreamAttrValue attr = {};
    attr.accessPolicyWindow = window;
    WETRIC_CUDA_TRY(cudaStreamSetAttribute(
        st, cudaStreamAttributeAccessPolicyWindow, &attr));
    window_set = true;
  }

  // Per-row hash sets for the rows outside the bitmap (kernels 6-8), their
  // buckets filled chunk by chunk below. Without room for them (or with
  // 2^32 buckets or more) the count searches the rows instead.
  Scratch<uint32_t> htab;
  Scratch<uint2> hrows;
  HashView hv{};
  if (want_hash && buckets && buckets < (1ull << 32)) {
    if (htab.alloc(ctx, st, buckets * kHashBucket) == WETRIC_OK &&
        hrows.alloc(ctx, st, n) == WETRIC_OK) {
      WETRIC_CUDA_TRY(cudaMemsetAsync(htab.ptr, 0xFF,
                                      buckets * kHashBucket * sizeof(uint32_t), st));
      k_hash_rows<<<grid_for(ctx, n), 256, 0, st>>>(hoff.ptr, n, hrows.ptr);
      WETRIC_LAUNCH_CHECK();
      ++launches;
      hv.rows = hrows.ptr;
      hv.tab = htab.ptr;
    } else {
      clear_error();
    }
  }
  Scratch<uint32_t> ntab;
  Scratch<uint2> nrows;
  if (ncount && nbuckets && nbuckets < (1ull << 32)) {
    if (ntab.alloc(ctx, st, nbuckets * kNearWords) == WETRIC_OK &&
        nrows.alloc(ctx, st, ncount) == WETRIC_OK) {
      WETRIC_CUDA_TRY(cudaMemsetAsync(ntab.ptr, 0xFF,
                                      nbuckets * kNearWords * sizeof(uint32_t), st));
      k_hash_rows<<<grid_for(ctx, ncount), 256, 0, st>>>(noff.ptr, ncount,
                                                          nrows.ptr);
      WETRIC_LAUNCH_CHECK();
      ++launches;
      hv.nrows = nrows.ptr;
      hv.ntab = ntab.ptr;
      hv.nfirst = (uint32_t)nfirst;
      hv.ncount = (uint32_t)ncount;
      // rows of the core matrix are checked there: no near sets for them
      if (aligned)
        hv.ncount = (uint32_t)(core_v0 > nfirst ? (core_v0 - nfirst < ncount ? core_v0 - nfirst
                                                                               : ncount)
                                                : 0);
    } else {
      clear_error();  // the near rows are searched instead
    }
  }

  // The core bit matrix, its rows written chunk by chunk below. The core
  // and shell kernels stage each vertex's row of columns in shared memory
  // by a TMA bulk copy when the column array is 16-byte aligned.
  Scratch<uint32_t> core;
  uint32_t core_H4 = 0;
  const bool tma_ok = (reinterpret_cast<uintptr_t>(a.col_ind) & 15) == 0;
  if (core_h) {
    core_H4 = (uint32_t)(4 * ceil_div(core_h, 128));
    const uint64_t cwords = core_row_off(core_H4, (uint32_t)core_h);
    WETRIC_TRY(core.alloc(ctx, st, cwords + 4));
    WETRIC_CUDA_TRY(cudaMemsetAsync(core.ptr, 0, (cwords + 4) * sizeof(uint32_t), st));
  }

  int occ = 0;
  uint64_t grid = 0;
  Scratch<unsigned long long> next_tile;
  // Warp kernels: 2 = warp-staged, 3 = row-walk with the shared-memory
  // stage, 4 = row-walk without it (the searches hit L1/L2 and the stage
  // only adds instructions), 5 = 4 built for 6 blocks per SM, 6 = 5 with
  // per-row hash sets for the rows outside the bitmap, 7 = 6 with long-row
  // segments at 5 blocks per SM (48 registers, no spills), 8 = 7 with
  // 16-bit near sets for the hash rows within 65536 of the end (48
  // registers, no spills; default: fastest measured on B200 at every
  // bitmap length tried).
  const void *warp_fn =
      kid == 2 ? (const void *)k_count_staged<Off, false>
      : kid == 4 ? (const void *)k_count_rows<Off, false, false>
      : kid == 5 ? (const void *)k_count_rows<Off, false, false, 6>
      : kid == 6 ? (const void *)k_count_rows<Off, false, false, 6, true>
      : kid == 7 ? (aligned ? (const void *)k_count_rows<Off, false, false, kSegsMinBlocks, true,
                                                         true, false, true>
                            : (const void *)k_count_rows<Off, false, false, kSegsMinBlocks, true,
                                                         true>)
      : kid == 8 ? (aligned ? (const void *)k_count_rows<Off, false, false, kSegsMinBlocks, true,
                                                         true, true, true>
                            : (const void *)k_count_rows<Off, false, false, kSegsMinBlocks, true,
                                                         true, true>)
                 : (const void *)k_count_rows<Off, false, true>;
  if (staged_kernel) {
    WETRIC_TRY(next_tile.alloc(ctx, st, C));
    WETRIC_CUDA_TRY(cudaMemsetAsync(next_tile.ptr, 0, C * sizeof(unsigned long long), st));
    WETRIC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &occ, warp_fn, (int)B, 0));
  } else {
    WETRIC_CUDA_TRY(cudaFuncSetAttribute(
        k_count<Off>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    WETRIC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &occ, k_count<Off>, (int)B, smem));
  }
  if (occ < 1) occ = 1;
  const uint64_t full_grid = (uint64_t)ctx->sm_count * occ;

  EventPair ev_chunk[kMaxColChunks], ev_core[kMaxColChunks], ev_shell[kMaxColChunks];
  double count_ms = 0.0, core_ms = 0.0, shell_ms = 0.0, pair_ms = 0.0;
  NvtxRange nvtx_launch("wetric count: structures and kernels");
  // Pair streams: tiles of up to kPairTile streamed columns (fewer for
  // small totals: about two tiles per warp slot of the device), one warp
  // per tile.
  EventPair ev_pair;
  Scratch<uint32_t> ptile;
  if (Rp) {
    const uint64_t Tp = pair_tile_cols(Rp, ctx->sm_count);
    const uint64_t ptiles = ceil_div(Rp, Tp);
    WETRIC_TRY(ps.alloc(ctx, st, Kp + 1));
    WETRIC_TRY((prim::exclusive_scan<uint32_t, uint64_t>(ctx, st, pl.ptr, ps.ptr, Kp)));
    WETRIC_TRY(ptile.alloc(ctx, st, ptiles + 1));
    k_tile_map<<<grid_for(ctx, ptiles + 1), 256, 0, st>>>(ps.ptr, Kp, 0, Rp, Tp, ptiles,
                                                          ptile.ptr);
    WETRIC_LAUNCH_CHECK();
    WETRIC_TRY(ev_pair.create());
    WETRIC_CUDA_TRY(cudaEventRecord(ev_pair.a, st));
    k_count_pairs<false><<<(unsigned)ceil_div(ptiles, kPairWarps), kPairWarps * 32, 0, st>>>(
        reinterpret_cast<const uint32_t *>(rp), a.col_ind, pv.ptr, ps.ptr, nullptr, Kp,
        ptile.ptr, ptiles, Tp, acc.ptr + 1, nullptr);
    WETRIC_LAUNCH_CHECK();
    WETRIC_CUDA_TRY(cudaEventRecord(ev_pair.b, st));
    launches += 5;
  }
  for (uint32_t i = 0; i < C; ++i) {
    const Chunk &c = ch[i];
    if (c.ready) WETRIC_CUDA_TRY(cudaStreamWaitEvent(st, c.ready, 0));
    // This chunk's bitmap rows and hash sets (every row above it is built).
    if (words) {
      const uint64_t b0 = c.lo > first_row ? c.lo : first_row;
      if (c.hi > b0) {
        k_bitmap<Off><<<grid_for(ctx, (c.hi - b0) * 32), 256, 0, st>>>(
            rp, a.col_ind, n, b0, S, bm.ptr, c.hi);
        WETRIC_LAUNCH_CHECK();
        ++launches;
      }
    }
    if (hv.rows) {
      k_hash_build<Off><<<grid_for(ctx, (c.hi - c.lo) * 32), 256, 0, st>>>(
          rp, a.col_ind, n, hoff.ptr, htab.ptr, c.lo, c.hi);
      WETRIC_LAUNCH_CHECK();
      ++launches;
    }
    if (hv.nrows && hv.ncount) {
      const uint64_t r0 = (c.lo > nfirst ? c.lo : nfirst) - nfirst;
      const uint64_t r1 = (c.hi < nfirst + hv.ncount ? c.hi : nfirst + hv.ncount);
      if (r1 > nfirst && r1 - nfirst > r0) {
        k_near_build<Off><<<grid_for(ctx, (r1 - nfirst - r0) * 32), 256, 0, st>>>(
            rp, a.col_ind, n, nfirst, r1 - nfirst, noff.ptr, ntab.ptr, r0);
        WETRIC_LAUNCH_CHECK();
        ++launches;
      }
    }
    if (core_h && c.hi > core_v0) {
      const uint64_t r0 = (c.lo > core_v0 ? c.lo : core_v0) - core_v0;
      const uint64_t r1 = c.hi - core_v0;
      k_core_bitmap<Off><<<grid_for(ctx, (r1 - r0) * 32), 256, 0, st>>>(
          rp, a.col_ind, core_v0, (uint32_t)core_h, core_H4, core.ptr, (uint32_t)r0,
          (uint32_t)r1);
      WETRIC_LAUNCH_CHECK();
      ++launches;
    }
    if (core_hi[i] > core_lo[i] && K > core_K) {
      WETRIC_TRY(ev_core[i].create());
      WETRIC_CUDA_TRY(cudaEventRecord(ev_core[i].a, st));
      k_core_count<Off><<<(unsigned)(K - core_K), kCoreBlock, 0, st>>>(
          a.col_ind, core.ptr, core_v0, (uint32_t)core_h, core_H4, act_wp.ptr,
          act_rb.ptr, act_d.ptr, core_K, K, core_lo[i], core_hi[i], acc.ptr + 1, tma_ok,
          small.ptr);
      WETRIC_LAUNCH_CHECK();
      ++launches;
      WETRIC_CUDA_TRY(cudaEventRecord(ev_core[i].b, st));
      r->core_wedges += core_hi[i] - core_lo[i];
    }
    if (shell_hi[i] > shell_lo[i] && core_K > shell_K) {
      WETRIC_TRY(ev_shell[i].create());
      WETRIC_CUDA_TRY(cudaEventRecord(ev_shell[i].a, st));
      if (kid == 8)
        k_shell_count<Off, true><<<(unsigned)(core_K - shell_K), kCoreBlock, 0, st>>>(
            rp, a.col_ind, n, core.ptr, core_v0, (uint32_t)core_h, core_H4, act_wp.ptr,
            act_rb.ptr, act_d.ptr, shell_K, core_K, shell_lo[i], shell_hi[i], hv, acc.ptr + 1,
            tma_ok, small.ptr);
      else
        k_shell_count<Off, false><<<(unsigned)(core_K - shell_K), kCoreBlock, 0, st>>>(
            rp, a.col_ind, n, core.ptr, core_v0, (uint32_t)core_h, core_H4, act_wp.ptr,
            act_rb.ptr, act_d.ptr, shell_K, core_K, shell_lo[i], shell_hi[i], hv, acc.ptr + 1,
            tma_ok, small.ptr);
      WETRIC_LAUNCH_CHECK();
      ++launches;
      WETRIC_CUDA_TRY(cudaEventRecord(ev_shell[i].b, st));
      r->shell_wedges += shell_hi[i] - shell_lo[i];
    }
    if (!c.tiles) continue;
    const uint32_t *tk = tile_k.ptr + c.toff;
    uint64_t g = full_grid;
    unsigned long long *counter = staged_kernel ? next_tile.ptr + i : nullptr;
    if (staged_kernel) {
      const uint64_t warps_needed = ceil_div(c.tiles, kWarpsPerBlock);
      if (g > warps_needed) g = warps_needed;
      if (!a.persistent && kid != 2 && warps_needed <= 0x7FFFFFFFull) {
        g = warps_needed;  // one warp per tile, no tile counter
        counter = nullptr;
      }
    } else if (g > c.tiles) {
      g = c.tiles;
    }
    if (g > grid) grid = g;
    WETRIC_TRY(ev_chunk[i].create());
    WETRIC_CUDA_TRY(cudaEventRecord(ev_chunk[i].a, st));
    if (staged_kernel) {
      if (kid == 2)
        k_count_staged<Off, false><<<(unsigned)g, B, 0, st>>>(
            rp, a.col_ind, n, act_wp.ptr, act_rb.ptr, act_d.ptr, K, tk,
            c.tiles, c.wlo, c.whi, T, bm.ptr, bm_first, S, next_tile.ptr + i,
            acc.ptr + 1, BatchView{});
      else if (kid == 4)
        k_count_rows<Off, false, false><<<(unsigned)g, B, 0, st>>>(
            rp, a.col_ind, n, act_wp.ptr, act_rb.ptr, act_d.ptr, K, tk,
            c.tiles, c.wlo, c.whi, T, bm.ptr, bm_first, S, counter,
            acc.ptr + 1, BatchView{});
      else if (kid == 5)
        k_count_rows<Off, false, false, 6><<<(unsigned)g, B, 0, st>>>(
            rp, a.col_ind, n, act_wp.ptr, act_rb.ptr, act_d.ptr, K, tk,
            c.tiles, c.wlo, c.whi, T, bm.ptr, bm_first, S, counter,
            acc.ptr + 1, BatchView{});
      else if (kid == 6)
        k_count_rows<Off, false, false, 6, true><<<(unsigned)g, B, 0, st>>>(
            rp, a.col_ind, n, act_wp.ptr, act_rb.ptr, act_d.ptr, K, tk,
            c.tiles, c.wlo, c.whi, T, bm.ptr, bm_first, S, counter,
            acc.ptr + 1, BatchView{}, hv);
      else if (kid == 7 && aligned)
        k_count_rows<Off, false, false, kSegsMinBlocks, true, true, false, true>
            <<<(unsigned)g, B, 0, st>>>(
                rp, a.col_ind, n, act_wp.ptr, act_rb.ptr, act_d.ptr, K, tk,
                c.tiles, c.wlo, c.whi, T, core.ptr, core_v0, core_H4, counter,
                acc.ptr + 1, BatchView{}, hv);
      else if (kid == 7)
        k_count_rows<Off, false, false, kSegsMinBlocks, true, true>
            <<<(unsigned)g, B, 0, st>>>(
                rp, a.col_ind, n, act_wp.ptr, act_rb.ptr, act_d.ptr, K, tk,
                c.tiles, c.wlo, c.whi, T, bm.ptr, bm_first, S, counter,
                acc.ptr + 1, BatchView{}, hv);
      else if (kid == 8 && aligned)
        k_count_rows<Off, false, false, kSegsMinBlocks, true, true, true, true>
            <<<(unsigned)g, B, 0, st>>>(
                rp, a.col_ind, n, act_wp.ptr, act_rb.ptr, act_d.ptr, K, tk,
                c.tiles, c.wlo, c.whi, T, core.ptr, core_v0, core_H4, counter,
                acc.ptr + 1, BatchView{}, hv);
      else if (kid == 8)
        k_count_rows<Off, false, false, kSegsMinBlocks, true, true, true>
            <<<(unsigned)g, B, 0, st>>>(
                rp, a.col_ind, n, act_wp.ptr, act_rb.ptr, act_d.ptr, K, tk,
                c.tiles, c.wlo, c.whi, T, bm.ptr, bm_first, S, counter,
                acc.ptr + 1, BatchView{}, hv);
      else
        k_count_rows<Off, false, true><<<(unsigned)g, B, 0, st>>>(
            rp, a.col_ind, n, act_wp.ptr, act_rb.ptr, act_d.ptr, K, tk,
            c.tiles, c.wlo, c.whi, T, bm.ptr, bm_first, S, counter,
            acc.ptr + 1, BatchView{});
    } else {
      k_count<Off><<<(unsigned)g, B, smem, st>>>(
          rp, a.col_ind, n, act_wp.ptr, act_rb.ptr, act_d.ptr, tk, c.tiles,
          c.wlo, c.whi, s, bm.ptr, bm_first, S, acc.ptr + 1);
    }
    WETRIC_LAUNCH_CHECK();
    ++launches;
    WETRIC_CUDA_TRY(cudaEventRecord(ev_chunk[i].b, st));
  }
  unsigned long long tri = 0;
  uint32_t err_after = 0;
  {
    ReadPlan rd;
    const uint32_t iT = rd.add(acc.ptr + 1, 1, 8), iE = rd.add(small.ptr, 1, 4);
    uint64_t local[kReadWords];
    const uint64_t *w = nullptr;
    WETRIC_TRY(read_back(ctx, st, rd, local, &w, ev_all.b));
    tri = w[iT];
    err_after = (uint32_t)w[iE];
  }
  if (window_set) {
    cudaStreamAttrValue attr = {};
    attr.accessPolicyWindow.num_bytes = 0;
    cudaStreamSetAttribute(st, cudaStreamAttributeAccessPolicyWindow, &attr);
    cudaCtxResetPersistingL2Cache();
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0);
  }
  float ms_all = 0;
  WETRIC_CUDA_TRY(cudaEventElapsedTime(&ms_all, ev_all.a, ev_all.b));
  for (uint32_t i = 0; i < C; ++i) {
    float ms = 0;
    if (ev_chunk[i].a) {
      WETRIC_CUDA_TRY(cudaEventElapsedTime(&ms, ev_chunk[i].a, ev_chunk[i].b));
      count_ms += ms;
    }
    if (ev_core[i].a) {
      WETRIC_CUDA_TRY(cudaEventElapsedTime(&ms, ev_core[i].a, ev_core[i].b));
      core_ms += ms;
    }
    if (ev_shell[i].a) {
      WETRIC_CUDA_TRY(cudaEventElapsedTime(&ms, ev_shell[i].a, ev_shell[i].b));
      shell_ms += ms;
    }
  }
  if (ev_pair.a) {
    float ms = 0;
    WETRIC_CUDA_TRY(cudaEventElapsedTime(&ms, ev_pair.a, ev_pair.b));
    pair_ms = ms;
  }
  if (err_after == kDevStageTimeout) {
    set_error(WETRIC_ETIMEDOUT, "a shared-memory staging copy did not complete in time");
    return WETRIC_ETIMEDOUT;
  }
  r->triangles = tri;
  r->exec_ms = ms_all;
  r->count_ms = count_ms + core_ms + shell_ms + pair_ms;
  r->pair_ms = pair_ms;
  r->core_ms = core_ms;
  r->shell_ms = shell_ms;
  r->block = B;
  r->grid = (uint32_t)grid;
  r->launches = launches;
  return WETRIC_OK;
}

}  // namespace

int count_oriented(DeviceContext *ctx, cudaStream_t st, const CountArgs &a,
                   CountResult *r) {
  if (a.spread == 0) {
    set_error(WETRIC_EINVAL, "spread must be > 0");
    return WETRIC_EINVAL;
  }
  if (a.bitmap_len % 32 != 0) {
    set_error(WETRIC_EINVAL, "bitmap length %u is not a multiple of 32",
              a.bitmap_len);
    return WETRIC_EINVAL;
  }
  if (a.n >= (1ull << 32)) {
    set_error(WETRIC_ERANGE, "n = %llu exceeds 2^32 - 1",
              (unsigned long long)a.n);
    return WETRIC_ERANGE;
  }
  if (a.offsets32 && a.m >= (1ull << 32)) {
    set_error(WETRIC_ERANGE, "u32 offsets with m >= 2^32");
    return WETRIC_ERANGE;
  }
  if (a.offsets32) return count_impl<uint32_t>(ctx, st, a, r);
  return count_impl<uint64_t>(ctx, st, a, r);
}

template <typename Off>
static int wedge_total_impl(DeviceContext *ctx, cudaStream_t st,
                            const Off *rp, uint64_t n, uint64_t *W,
                            uint64_t *maxdeg) {
  Scratch<uint32_t> active;
  Scratch<uint64_t> wc;
  Scratch<unsigned long long> md;
  Scratch<uint32_t> err;
  WETRIC_TRY(active.alloc(ctx, st, n));
  WETRIC_TRY(wc.alloc(ctx, st, n + 1));
  WETRIC_TRY(md.alloc(ctx, st, 1));
  WETRIC_TRY(err.alloc(ctx, st, 1));
  WETRIC_CUDA_TRY(cudaMemsetAsync(md.ptr, 0, sizeof(unsigned long long), st));
  WETRIC_CUDA_TRY(cudaMemsetAsync(err.ptr, 0, sizeof(uint32_t), st));
  uint64_t m = 0;
  if (n > 0) {
    Off last = 0;
    WETRIC_CUDA_TRY(cudaMemcpyAsync(&last, rp + n, sizeof(Off),
                                    cudaMemcpyDeviceToHost, st));
    WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
    m = last;
    k_vertex_wedges<Off><<<grid_for(ctx, n), 256, 0, st>>>(
        rp, n, m, active.ptr, md.ptr, err.ptr);
    WETRIC_LAUNCH_CHECK();
    // Reuse: wc[v] = C(d, 2) for all v (compact with pos == identity).
    WETRIC_TRY((prim::exclusive_scan<uint32_t, uint64_t>(ctx, st, active.ptr,
                                                         wc.ptr, n)));
  }
  uint64_t K = 0;
  uint32_t herr = 0;
  if (n > 0)
    WETRIC_CUDA_TRY(cudaMemcpyAsync(&K, wc.ptr + n, sizeof(uint64_t),
                                    cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(&herr, err.ptr, sizeof(uint32_t),
                                  cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  if (herr != kDevOk) {
    set_error(WETRIC_EINVAL, "row offsets check failed (device code %u)", herr);
    return WETRIC_EINVAL;
  }
  Scratch<uint64_t> act_wp, act_rb;
  Scratch<uint32_t> act_d;
  WETRIC_TRY(act_wp.alloc(ctx, st, K + 1));
  WETRIC_TRY(act_rb.alloc(ctx, st, K));
  WETRIC_TRY(act_d.alloc(ctx, st, K));
  if (K > 0) {
    k_compact_active<Off><<<grid_for(ctx, n), 256, 0, st>>>(
        rp, n, active.ptr, wc.ptr, act_wp.ptr, act_rb.ptr, act_d.ptr);
    WETRIC_LAUNCH_CHECK();
  }
  WETRIC_TRY((prim::exclusive_scan<uint64_t, uint64_t>(ctx, st, act_wp.ptr,
                                                       act_wp.ptr, K)));
  unsigned long long hmd = 0;
  WETRIC_CUDA_TRY(cudaMemcpyAsync(W, act_wp.ptr + K, sizeof(uint64_t),
                                  cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(&hmd, md.ptr, sizeof(hmd),
                                  cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  *maxdeg = hmd;
  return WETRIC_OK;
}

int wedge_total(DeviceContext *ctx, cudaStream_t st, const void *row_ptr,
                bool offsets32, uint64_t n, uint64_t *W, uint64_t *maxdeg) {
  if (offsets32)
    return wedge_total_impl<uint32_t>(
        ctx, st, static_cast<const uint32_t *>(row_ptr), n, W, maxdeg);
  return wedge_total_impl<uint64_t>(
      ctx, st, static_cast<const uint64_t *>(row_ptr), n, W, maxdeg);
}

int algorithmic_bytes(DeviceContext *ctx, cudaStream_t st, const void *row_ptr,
                      bool offsets32, const uint32_t *col_ind, uint64_t n,
                      uint64_t m, uint64_t *bytes) {
  Scratch<unsigned long long> acc;
  WETRIC_TRY(acc.alloc(ctx, st, 1));
  WETRIC_CUDA_TRY(cudaMemsetAsync(acc.ptr, 0, sizeof(unsigned long long), st));
  if (n > 0) {
    if (offsets32)
      k_alg_bytes<uint32_t><<<grid_for(ctx, n * 32), 256, 0, st>>>(
          static_cast<const uint32_t *>(row_ptr), col_ind, n, m, acc.ptr);
    else
      k_alg_bytes<uint64_t><<<grid_for(ctx, n * 32), 256, 0, st>>>(
          static_cast<const uint64_t *>(row_ptr), col_ind, n, m, acc.ptr);
    WETRIC_LAUNCH_CHECK();
  }
  unsigned long long h = 0;
  WETRIC_CUDA_TRY(cudaMemcpyAsync(&h, acc.ptr, sizeof(h),
                                  cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  // Streamed once: u64 row offsets, columns, u64 wedge prefix.
  *bytes = h + 8 * (n + 1) + 4 * m + 8 * (n + 1);
  return WETRIC_OK;
}

int narrow_offsets(DeviceContext *ctx, cudaStream_t st, const uint64_t *rp64,
                   uint64_t n, uint32_t *rp32) {
  k_narrow<<<grid_for(ctx, n + 1), 256, 0, st>>>(rp64, n, rp32);
  WETRIC_LAUNCH_CHECK();
  return WETRIC_OK;
}

int widen_offsets(DeviceContext *ctx, cudaStream_t st, const uint32_t *rp32,
                  uint64_t n, uint64_t *rp64) {
  k_widen<<<grid_for(ctx, n + 1), 256, 0, st>>>(rp32, n, rp64);
  WETRIC_LAUNCH_CHECK();
  return WETRIC_OK;
}

}  // namespace wetric
