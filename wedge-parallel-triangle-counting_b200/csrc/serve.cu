// serve.cu -- the resident serving engine.
//
// The reference has no serving layer (one graph per process run,
// tc.cu:816-918). Here one persistent kernel (k_serve) stays on the device
// and counts tiles of whichever requests the host has published:
//   * a request is preprocessed on a lane stream (orientation, then
//     serve_prepare: every structure of the row-walk count) while the
//     resident kernel runs -- it is launched with fewer blocks per SM than
//     fit, so the preprocessing kernels get SMs beside it;
//   * it is registered in a slot (the slot table in device memory holds its
//     pointers and sizes) and its tiles are published as queue items in
//     host-mapped memory; the kernel's warps take items in order, claim
//     tiles of the head item with a per-item counter, count each tile with
//     the same device code as the single-graph count (rows_tile), and the
//     warp that completes a slot's last tile writes the slot's count to
//     host-mapped memory, where the host sees it without synchronising;
//   * every wait of the kernel is bounded: a warp that finds the queue
//     empty for idle_us gives up, every other warp follows after its
//     current tile, and the kernel ends with status kServeIdle (the host
//     relaunches it when work arrives); a stop flag drains it.
// The warp that moves the queue head past an item sets that item's flag in
// host-mapped memory; the host counts the items taken by scanning the flags
// in order (stores of different warps may reach the host out of order, so
// a single head value written by whichever warp moved it last could go
// backwards on the host).
// The count's loads go through the non-coherent cache, which must not see
// memory change under a running kernel, so a completed request's memory is
// retired and freed only while no resident kernel runs; slots and items are
// numbered within a sequence space and never reused inside it. What does
// change under a running kernel -- the queue, the slot table as requests
// are registered -- is read through L2 (volatile loads, __ldcg).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <atomic>
#include <chrono>

#include "count.cuh"
#include "count_kernels.cuh"
#include "pair_streams.cuh"
#include "primitives.cuh"
#include "serve.cuh"

namespace wetric {

namespace {

unsigned grid_for(DeviceContext *ctx, uint64_t work, uint32_t block = 256) {
  const uint64_t cap = (uint64_t)ctx->sm_count * 32;
  uint64_t g = ceil_div(work, block);
  if (g > cap) g = cap;
  if (g == 0) g = 1;
  return (unsigned)g;
}

// One request as the resident kernel sees it (device memory, written once
// per sequence space before the request's first item is published).
struct ServeGraph {
  const uint32_t *rp;
  const uint32_t *ci;
  uint64_t n;
  const uint64_t *act_wp;
  const uint64_t *act_rb;
  const uint32_t *act_d;
  uint64_t K;
  const uint32_t *tile_k;
  uint64_t tiles, W, T;
  const uint32_t *bm;
  uint64_t bm_first, S;
  HashView hv;
};

// A queue item: tiles [t_begin, t_end) of one slot. Items and the tail
// live in device memory; the host publishes an item with two copies on one
// stream -- the item, then the new tail -- so the kernel sees the item
// before the tail that covers it, and its per-tile polling stays in L2.
struct ServeItem {
  uint32_t slot, pad;
  uint64_t t_begin, t_end, pad2;
};

enum ServeExit : uint32_t { kServeRunning = 0, kServeStopped = 1, kServeIdle = 2 };

constexpr uint32_t kServeMaxBlocksPerSm = 4;

__device__ __forceinline__ void st_release_sys(volatile unsigned long long *p,
                                               unsigned long long v) {
  asm volatile("st.release.sys.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void st_release_sys32(volatile uint32_t *p, uint32_t v) {
  asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// A slot's record, read through L2 (not the non-coherent L1 path): the
// slot table is written while the kernel runs (a new request's slot next to
// the slots already counting), and an L1 line that holds part of a slot read
// earlier could hold the next slot's record from before it was written.
__device__ __forceinline__ ServeGraph load_graph(const ServeGraph *p) {
  static_assert(sizeof(ServeGraph) % 8 == 0, "slot records are whole 8-byte words");
  ServeGraph g;
  const unsigned long long *src = reinterpret_cast<const unsigned long long *>(p);
  unsigned long long *dst = reinterpret_cast<unsigned long long *>(&g);
#pragma unroll
  for (int i = 0; i < (int)(sizeof(ServeGraph) / 8); ++i) dst[i] = __ldcg(src + i);
  return g;
}

template <bool kNear>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, kServeMaxBlocksPerSm)
    k_serve(const ServeGraph *graphs, const volatile ServeItem *items,
            const volatile unsigned long long *tail, const volatile uint32_t *stop_host,
            unsigned long long *head, unsigned long long *item_next,
            unsigned long long *slot_count, unsigned long long *slot_tiles,
            volatile unsigned long long *done_host,
            volatile uint32_t *passed_host, uint32_t *exit_code,
            unsigned long long idle_ns) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t why = kServeRunning;
  unsigned long long idle_since = 0;
  bool idle = false;
  // exit_code[1]: set by the first warp whose bounded wait runs out; every
  // warp then leaves after its current tile, so the kernel ends as a whole
  // and the host relaunches it for new work (warps that left one by one
  // would leave the queue to the few still busy)
  volatile uint32_t *quit = exit_code + 1;
  for (;;) {
    unsigned long long h = 0, tl = 0;
    uint32_t q = 0;
    if (lane == 0) {
      h = *reinterpret_cast<volatile unsigned long long *>(head);
      tl = *tail;
      q = *quit;
    }
    h = __shfl_sync(0xffffffffu, h, 0);
    tl = __shfl_sync(0xffffffffu, tl, 0);
    q = __shfl_sync(0xffffffffu, q, 0);
    if (q) {
      why = kServeIdle;
      break;
    }
    if (h >= tl) {
      // only an empty queue reads the host's stop flag (host memory)
      uint32_t st = 0;
      if (lane == 0) st = *stop_host;
      st = __shfl_sync(0xffffffffu, st, 0);
      if (st) {
        why = kServeStopped;
        break;
      }
      // Bounded wait: give up after idle_ns of an empty queue.
      unsigned long long now = 0;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
      if (!idle) {
        idle = true;
        idle_since = now;
      } else if (now - idle_since > idle_ns) {
        if (lane == 0) atomicExch(exit_code + 1, 1u);
        why = kServeIdle;
        break;
      }
      __nanosleep(2000);
      continue;
    }
    idle = false;
    uint32_t slot = 0;
    unsigned long long t0 = 0, t1 = 0, t = 0;
    if (lane == 0) {
      slot = items[h].slot;
      t0 = items[h].t_begin;
      t1 = items[h].t_end;
      t = t0 + atomicAdd(item_next + h, 1ull);
    }
    slot = __shfl_sync(0xffffffffu, slot, 0);
    t1 = __shfl_sync(0xffffffffu, t1, 0);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= t1) {
      // item h is used up: move the head past it (one warp succeeds)
      if (lane == 0 && atomicCAS(head, h, h + 1) == h) st_release_sys32(passed_host + h, 1u);
      continue;
    }
    const ServeGraph g = load_graph(graphs + slot);
    uint64_t acc = 0, staged = ~0ull;
    uint32_t staged_d = 0, cur_g = 0xFFFFFFFFu;
    rows_tile<uint32_t, false, false, true, true, kNear>(
        g.rp, g.ci, g.n, g.act_wp, g.act_rb, g.act_d, g.K, g.tile_k, t, 0, g.W, g.T,
        g.bm, g.bm_first, g.S, BatchView{}, g.hv, nullptr, staged, staged_d, acc, cur_g);
    const uint32_t tot = __reduce_add_sync(0xffffffffu, (uint32_t)acc);
    if (lane == 0) {
      if (tot) atomicAdd(slot_count + slot, (unsigned long long)tot);
      __threadfence();
      const unsigned long long done = atomicAdd(slot_tiles + slot, 1ull) + 1;
      if (done == g.tiles) {
        __threadfence();
        const unsigned long long total = atomicAdd(slot_count + slot, 0ull);
        st_release_sys(done_host + slot, total + 1);
      }
    }
  }
  if (lane == 0) atomicMax(exit_code, why);
}

void *host_mapped(size_t bytes, void **dev) {
  void *h = nullptr;
  if (cudaHostAlloc(&h, bytes, cudaHostAllocMapped) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  memset(h, 0, bytes);
  if (cudaHostGetDevicePointer(dev, h, 0) != cudaSuccess) {
    cudaGetLastError();
    cudaFreeHost(h);
    return nullptr;
  }
  return h;
}

}  // namespace

// ------------------------------------------------------------ preparation

int serve_prepare(DeviceContext *ctx, cudaStream_t st, uint32_t spread,
                  uint32_t bitmap_len, ServePlan *p) {
  NvtxRange nvtx_("wetric serve prepare");
  if (spread == 0 || bitmap_len % 32 != 0) {
    set_error(WETRIC_EINVAL, "bad spread or bitmap length");
    return WETRIC_EINVAL;
  }
  const uint64_t n = p->csr.n, m = p->csr.m;
  p->n = n;
  p->m = m;
  if (m >= (1ull << 32)) {
    set_error(WETRIC_ERANGE, "served graphs need m < 2^32");
    return WETRIC_ERANGE;
  }
  if (n == 0) return WETRIC_OK;
  // u32 offsets for the count
  WETRIC_TRY(p->rp32.alloc(ctx, st, n + 1));
  WETRIC_TRY(narrow_offsets(ctx, st, p->csr.row_ptr, n, p->rp32.ptr));
  const uint32_t *rp = p->rp32.ptr;
  const uint32_t *ci = p->csr.col_ind;
  Scratch<uint32_t> small, active, nb;
  Scratch<unsigned long long> acc;
  Scratch<uint64_t> pos, hoff, noff;
  WETRIC_TRY(small.alloc(ctx, st, 4));
  WETRIC_TRY(acc.alloc(ctx, st, 5));
  WETRIC_CUDA_TRY(cudaMemsetAsync(small.ptr, 0, 4 * sizeof(uint32_t), st));
  WETRIC_CUDA_TRY(cudaMemsetAsync(acc.ptr, 0, 5 * sizeof(unsigned long long), st));
  WETRIC_TRY(active.alloc(ctx, st, n));
  WETRIC_TRY(pos.alloc(ctx, st, n + 1));
  k_vertex_wedges<uint32_t><<<grid_for(ctx, n), 256, 0, st>>>(rp, n, m, active.ptr,
                                                              acc.ptr, small.ptr);
  WETRIC_LAUNCH_CHECK();
  // Pair streams for the short rows (as count_oriented): they leave the
  // resident kernel's active set.
  Scratch<uint32_t> pl;
  const bool pairs = m >= kPairMinColumns;
  if (pairs) {
    WETRIC_TRY(p->pv.alloc(ctx, st, n));
    WETRIC_TRY(pl.alloc(ctx, st, n));
    k_pair_plan<<<grid_for(ctx, n), 256, 0, st>>>(rp, ci, n, active.ptr, p->pv.ptr, pl.ptr,
                                                  acc.ptr + 2);
    WETRIC_LAUNCH_CHECK();
  }
  WETRIC_TRY((prim::exclusive_scan<uint32_t, uint64_t>(ctx, st, active.ptr, pos.ptr, n)));
  WETRIC_TRY(p->act_wp.alloc(ctx, st, n + 1));
  WETRIC_TRY(p->act_rb.alloc(ctx, st, n));
  WETRIC_TRY(p->act_d.alloc(ctx, st, n));
  WETRIC_CUDA_TRY(cudaMemsetAsync(p->act_wp.ptr, 0, (n + 1) * sizeof(uint64_t), st));
  k_compact_active<uint32_t><<<grid_for(ctx, n), 256, 0, st>>>(
      rp, n, active.ptr, pos.ptr, p->act_wp.ptr, p->act_rb.ptr, p->act_d.ptr);
  WETRIC_LAUNCH_CHECK();
  WETRIC_TRY((prim::exclusive_scan<uint64_t, uint64_t>(ctx, st, p->act_wp.ptr,
                                                       p->act_wp.ptr, n)));
  // Edge-check structures of kernel 8: bitmap over the last a vertices,
  // 16-bit near sets for the rows with d+ >= 16 within 65536 of the end,
  // 32-bit hash sets for the other rows with d+ >= 16.
  const uint64_t alen = bitmap_len;
  const uint64_t bm_first = (n > alen ? n : alen) - alen;
  const uint64_t nfirst = (n > kNearSpan ? n : kNearSpan) - kNearSpan;
  const uint64_t ncount = nfirst < bm_first ? bm_first - nfirst : 0;
  WETRIC_TRY(nb.alloc(ctx, st, n));
  WETRIC_TRY(hoff.alloc(ctx, st, n + 1));
  k_hash_sizes<uint32_t><<<grid_for(ctx, n), 256, 0, st>>>(
      rp, n, ncount ? nfirst : bm_first, kHashMinDegree, kHashKeysPerBucket, nb.ptr);
  WETRIC_LAUNCH_CHECK();
  WETRIC_TRY((prim::exclusive_scan<uint32_t, uint64_t>(ctx, st, nb.ptr, hoff.ptr, n)));
  if (ncount) {
    WETRIC_TRY(noff.alloc(ctx, st, ncount + 1));
    k_hash_sizes<uint32_t><<<grid_for(ctx, ncount), 256, 0, st>>>(
        rp + nfirst, ncount, ncount, kHashMinDegree, kNearKeysPerBucket, nb.ptr);
    WETRIC_LAUNCH_CHECK();
    WETRIC_TRY((prim::exclusive_scan<uint32_t, uint64_t>(ctx, st, nb.ptr, noff.ptr, ncount)));
  }
  // Dense core and shell (as count_oriented): candidate sizes from the row
  // offsets and the first core / shell wedge of each, in the same read-back.
  Scratch<unsigned long long> cplan;
  Scratch<uint64_t> cstart;
  CoreStarts cs{};
  const bool core_ok = n >= 64;
  if (core_ok) {
    WETRIC_TRY(cplan.alloc(ctx, st, 2 * kCoreNumCandidates));
    WETRIC_CUDA_TRY(cudaMemsetAsync(cplan.ptr, 0,
                                    2 * kCoreNumCandidates * sizeof(unsigned long long), st));
    const uint64_t top = n < core_candidate(0) ? n : core_candidate(0);
    k_core_plan<uint32_t><<<grid_for(ctx, top), 256, 0, st>>>(rp, n, cplan.ptr);
    WETRIC_LAUNCH_CHECK();
    for (uint32_t c = 0; c < kCoreNumCandidates; ++c) {
      const uint64_t h = n < core_candidate(c) ? n : core_candidate(c);
      cs.v0[cs.c++] = n - h;
      cs.v0[cs.c++] = n - h;  // no shell: the wedge checks are faster there
    }
    WETRIC_TRY(cstart.alloc(ctx, st, 2 * cs.c));
    k_core_prefix<<<1, 32, 0, st>>>(p->act_wp.ptr, pos.ptr, cs, cstart.ptr);
    WETRIC_LAUNCH_CHECK();
  }
  unsigned long long plan[2 * kCoreNumCandidates] = {};
  uint64_t starts[2 * (2 * kCoreNumCandidates + 2)] = {};
  uint64_t K = 0, W = 0, buckets = 0, nbuckets = 0;
  unsigned long long maxdeg = 0;
  unsigned long long pacc[3] = {0, 0, 0};  // pair vertices, wedges, columns
  uint32_t err = 0;
  if (pairs)
    WETRIC_CUDA_TRY(cudaMemcpyAsync(pacc, acc.ptr + 2, sizeof(pacc), cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(&K, pos.ptr + n, 8, cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(&W, p->act_wp.ptr + n, 8, cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(&maxdeg, acc.ptr, 8, cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(&err, small.ptr, 4, cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(&buckets, hoff.ptr + n, 8, cudaMemcpyDeviceToHost, st));
  if (ncount)
    WETRIC_CUDA_TRY(cudaMemcpyAsync(&nbuckets, noff.ptr + ncount, 8,
                                    cudaMemcpyDeviceToHost, st));
  if (core_ok) {
    WETRIC_CUDA_TRY(cudaMemcpyAsync(plan, cplan.ptr, sizeof(plan), cudaMemcpyDeviceToHost, st));
    WETRIC_CUDA_TRY(cudaMemcpyAsync(starts, cstart.ptr, 2 * cs.c * sizeof(uint64_t),
                                    cudaMemcpyDeviceToHost, st));
  }
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  if (err != kDevOk) {
    set_error(WETRIC_EINVAL, "oriented CSR check failed (device code %u)", err);
    return WETRIC_EINVAL;
  }
  if (maxdeg >= kMaxOutDegree) {
    set_error(WETRIC_ERANGE, "max out-degree %llu >= 2^30", maxdeg);
    return WETRIC_ERANGE;
  }
  p->K = K;
  p->W = W;
  p->max_out_degree = maxdeg;
  const uint64_t Kp = pacc[0], Rp = pacc[2];
  p->pair_rows = Kp;
  p->pair_wedges = pacc[1];
  active.release();
  pos.release();
  nb.release();
  if (Rp) {
    WETRIC_TRY(p->ps.alloc(ctx, st, Kp + 1));
    WETRIC_TRY((prim::exclusive_scan<uint32_t, uint64_t>(ctx, st, pl.ptr, p->ps.ptr, Kp)));
  }
  pl.release();
  if (W == 0 && !Rp) return WETRIC_OK;
  // The core: count_oriented's rule (core_pick), with the shell below it
  // when the core covers the bitmap's rows.
  uint64_t core_h = 0, core_v0 = n, core_K = 0, core_W = W;
  uint64_t shell_K = 0, shell_W = W;
  const int c = core_ok ? core_pick(plan) : -1;
  if (c >= 0) {
    core_v0 = cs.v0[2 * c];
    core_h = n - core_v0;
    core_K = starts[4 * c];
    core_W = starts[4 * c + 1];
    shell_K = starts[4 * c + 2];
    shell_W = starts[4 * c + 3];
  }
  if (core_h < 32) {
    core_h = 0;
    core_W = shell_W = W;
  } else if (core_h < alen) {
    shell_K = core_K;
    shell_W = core_W;
  }
  // Tiles of 256 s wedges, smaller for small counts (about two per warp
  // slot of the device), as in count_oriented.
  uint64_t T = 256ull * spread;
  const uint64_t min_tiles = 2ull * (uint64_t)ctx->sm_count * 64;
  if (ceil_div(W, T) < min_tiles) {
    const uint64_t t = ceil_div(ceil_div(W, min_tiles), 32) * 32;
    T = t < T ? (t < 32 ? 32 : t) : T;
  }
  // The resident kernel's tiles: the wedges below the shell.
  p->T = T;
  p->W = shell_W;
  p->tiles = shell_W ? ceil_div(shell_W, T) : 0;
  WETRIC_TRY(p->tile_k.alloc(ctx, st, p->tiles + 1));
  if (p->tiles) {
    k_tile_map<<<grid_for(ctx, p->tiles + 1), 256, 0, st>>>(p->act_wp.ptr, K, 0, shell_W, T,
                                                            p->tiles, p->tile_k.ptr);
    WETRIC_LAUNCH_CHECK();
  }
  const uint64_t S = alen * (alen ? alen - 1 : 0) / 2;
  const uint64_t words = ceil_div(S, 32);
  const uint64_t first_row = n - (n < alen ? n : alen);
  p->S = S;
  p->bm_first = bm_first;
  WETRIC_TRY(p->bm.alloc(ctx, st, words ? words : 1));
  if (words) {
    WETRIC_CUDA_TRY(cudaMemsetAsync(p->bm.ptr, 0, words * sizeof(uint32_t), st));
    k_bitmap<uint32_t><<<grid_for(ctx, (n - first_row) * 32), 256, 0, st>>>(
        rp, ci, n, first_row, S, p->bm.ptr, n);
    WETRIC_LAUNCH_CHECK();
  }
  if (buckets && buckets < (1ull << 32) &&
      p->htab.alloc(ctx, st, buckets * kHashBucket) == WETRIC_OK &&
      p->hrows.alloc(ctx, st, n) == WETRIC_OK) {
    WETRIC_CUDA_TRY(cudaMemsetAsync(p->htab.ptr, 0xFF,
                                    buckets * kHashBucket * sizeof(uint32_t), st));
    k_hash_rows<<<grid_for(ctx, n), 256, 0, st>>>(hoff.ptr, n, p->hrows.ptr);
    WETRIC_LAUNCH_CHECK();
    k_hash_build<uint32_t><<<grid_for(ctx, n * 32), 256, 0, st>>>(rp, ci, n, hoff.ptr,
                                                                  p->htab.ptr);
    WETRIC_LAUNCH_CHECK();
  } else {
    clear_error();  // rows are searched instead
    p->htab.release();
  }
  if (ncount && nbuckets && nbuckets < (1ull << 32) &&
      p->ntab.alloc(ctx, st, nbuckets * kNearWords) == WETRIC_OK &&
      p->nrows.alloc(ctx, st, ncount) == WETRIC_OK) {
    WETRIC_CUDA_TRY(cudaMemsetAsync(p->ntab.ptr, 0xFF,
                                    nbuckets * kNearWords * sizeof(uint32_t), st));
    k_hash_rows<<<grid_for(ctx, ncount), 256, 0, st>>>(noff.ptr, ncount, p->nrows.ptr);
    WETRIC_LAUNCH_CHECK();
    k_near_build<uint32_t><<<grid_for(ctx, ncount * 32), 256, 0, st>>>(
        rp, ci, n, nfirst, ncount, noff.ptr, p->ntab.ptr, 0);
    WETRIC_LAUNCH_CHECK();
    p->nfirst = (uint32_t)nfirst;
    p->ncount = (uint32_t)ncount;
  } else {
    clear_error();
    p->ntab.release();
  }
  // Core matrix, then the core and shell counts on this stream (they run
  // beside the resident kernel; the plan is complete before they start).
  uint32_t core_H4 = 0;
  if (core_h || Rp) {
    WETRIC_TRY(p->core_acc.alloc(ctx, st, 1));
    WETRIC_CUDA_TRY(cudaMemsetAsync(p->core_acc.ptr, 0, 8, st));
  }
  if (core_h) {
    core_H4 = (uint32_t)(4 * ceil_div(core_h, 128));
    const uint64_t cwords = core_row_off(core_H4, (uint32_t)core_h) + 4;
    WETRIC_TRY(p->core.alloc(ctx, st, cwords));
    WETRIC_CUDA_TRY(cudaMemsetAsync(p->core.ptr, 0, cwords * 4, st));
    k_core_bitmap<uint32_t><<<grid_for(ctx, core_h * 32), 256, 0, st>>>(
        rp, ci, core_v0, (uint32_t)core_h, core_H4, p->core.ptr, 0, (uint32_t)core_h);
    WETRIC_LAUNCH_CHECK();
  }
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  if (core_h) {
    HashView hv{};
    if (p->htab.ptr) {
      hv.rows = p->hrows.ptr;
      hv.tab = p->htab.ptr;
    }
    if (p->ntab.ptr) {
      hv.nrows = p->nrows.ptr;
      hv.ntab = p->ntab.ptr;
      hv.nfirst = p->nfirst;
      hv.ncount = p->ncount;
    }
    if (K > core_K) {
      k_core_count<uint32_t><<<(unsigned)(K - core_K), kCoreBlock, 0, st>>>(
          ci, p->core.ptr, core_v0, (uint32_t)core_h, core_H4, p->act_wp.ptr, p->act_rb.ptr,
          p->act_d.ptr, core_K, K, core_W, W, p->core_acc.ptr);
      WETRIC_LAUNCH_CHECK();
    }
    if (core_K > shell_K) {
      k_shell_count<uint32_t, true><<<(unsigned)(core_K - shell_K), kCoreBlock, 0, st>>>(
          rp, ci, n, p->core.ptr, core_v0, (uint32_t)core_h, core_H4, p->act_wp.ptr,
          p->act_rb.ptr, p->act_d.ptr, shell_K, core_K, shell_W, core_W, hv, p->core_acc.ptr);
      WETRIC_LAUNCH_CHECK();
    }
    p->core_len = core_h;
    p->core_wedges = W - shell_W;
  }
  if (Rp) {
    // the pair streams: tiles of up to kPairTile streamed columns
    const uint64_t Tp = pair_tile_cols(Rp, ctx->sm_count);
    const uint64_t ptiles = ceil_div(Rp, Tp);
    WETRIC_TRY(p->ptile_k.alloc(ctx, st, ptiles + 1));
    k_tile_map<<<grid_for(ctx, ptiles + 1), 256, 0, st>>>(p->ps.ptr, Kp, 0, Rp, Tp, ptiles,
                                                          p->ptile_k.ptr);
    WETRIC_LAUNCH_CHECK();
    k_count_pairs<false><<<(unsigned)ceil_div(ptiles, kPairWarps), kPairWarps * 32, 0, st>>>(
        rp, ci, p->pv.ptr, p->ps.ptr, nullptr, Kp, p->ptile_k.ptr, ptiles, Tp,
        p->core_acc.ptr, nullptr);
    WETRIC_LAUNCH_CHECK();
  }
  if (core_h || Rp) {
    WETRIC_CUDA_TRY(cudaEventCreateWithFlags(&p->core_done, cudaEventDisableTiming));
    WETRIC_CUDA_TRY(cudaEventRecord(p->core_done, st));
  }
  p->bytes = p->csr.n * 8 + p->csr.m * 4 + p->rp32.bytes + p->act_wp.bytes +
             p->act_rb.bytes + p->act_d.bytes + p->tile_k.bytes + p->bm.bytes +
             p->htab.bytes + p->ntab.bytes + p->hrows.bytes + p->nrows.bytes + p->core.bytes +
             p->pv.bytes + p->ps.bytes + p->ptile_k.bytes;
  return WETRIC_OK;
}

// ----------------------------------------------------------------- engine

struct ServeEngine {
  DeviceContext *ctx = nullptr;
  ServeEngineOptions opt;
  cudaStream_t kstream = nullptr;  // the resident kernel
  cudaStream_t cstream = nullptr;  // slot-table writes
  // the queue: items and tail in device memory, published from pinned
  // host copies (one source slot per item and per tail value, so a later
  // publish cannot overwrite a source an earlier copy has yet to read)
  ServeItem *items_h = nullptr, *items_d = nullptr;
  unsigned long long *tail_src = nullptr, *tail_d = nullptr;
  // host-mapped control (host pointer / device pointer)
  unsigned long long *ctl_h = nullptr, *ctl_d = nullptr;
  uint32_t *stop_h = nullptr, *stop_d = nullptr;
  unsigned long long *done_h = nullptr, *done_d = nullptr;
  // one flag per item, set when the queue head has moved past it
  uint32_t *passed_h = nullptr, *passed_d = nullptr;
  // device state
  ServeGraph *graphs = nullptr;
  unsigned long long *head = nullptr, *item_next = nullptr, *slot_count = nullptr,
                     *slot_tiles = nullptr;
  uint32_t *exit_code = nullptr;
  int grid = 0;
  std::mutex mu;
  bool running = false;
  cudaEvent_t ended = nullptr;
  uint64_t published = 0, taken = 0;
  uint32_t next_slot = 0;
  std::vector<std::unique_ptr<ServePlan>> active;  // by slot (this space)
  std::vector<uint32_t> pending;                   // slots not yet completed
  std::vector<std::unique_ptr<ServePlan>> retired;
  uint64_t retired_bytes = 0, freed_bytes = 0, launches = 0, launch_errors = 0;
  uint32_t launch_error_code = 0;
  uint32_t last_exit = 0;
};

namespace {

int engine_reset_space(ServeEngine *e) {
  const ServeEngineOptions &o = e->opt;
  WETRIC_CUDA_TRY(cudaMemsetAsync(e->head, 0, sizeof(unsigned long long), e->cstream));
  WETRIC_CUDA_TRY(cudaMemsetAsync(e->tail_d, 0, sizeof(unsigned long long), e->cstream));
  WETRIC_CUDA_TRY(cudaMemsetAsync(e->item_next, 0, o.max_items * sizeof(unsigned long long),
                                  e->cstream));
  WETRIC_CUDA_TRY(cudaMemsetAsync(e->slot_count, 0, o.max_slots * sizeof(unsigned long long),
                                  e->cstream));
  WETRIC_CUDA_TRY(cudaMemsetAsync(e->slot_tiles, 0, o.max_slots * sizeof(unsigned long long),
                                  e->cstream));
  WETRIC_CUDA_TRY(cudaStreamSynchronize(e->cstream));
  memset(e->done_h, 0, o.max_slots * sizeof(unsigned long long));
  memset(e->passed_h, 0, o.max_items * sizeof(uint32_t));
  std::atomic_thread_fence(std::memory_order_seq_cst);
  e->published = 0;
  e->taken = 0;
  e->next_slot = 0;
  e->active.clear();
  e->active.resize(o.max_slots);
  e->pending.clear();
  return WETRIC_OK;
}

// Items the kernel has moved its head past: the longest prefix of set flags.
uint64_t engine_taken(ServeEngine *e) {
  const volatile uint32_t *f = e->passed_h;
  while (e->taken < e->published && f[e->taken]) ++e->taken;
  std::atomic_thread_fence(std::memory_order_acquire);
  return e->taken;
}

// Frees retired plans; only while no resident kernel runs.
void engine_free_retired(ServeEngine *e) {
  e->retired.clear();
  e->freed_bytes += e->retired_bytes;
  e->retired_bytes = 0;
}

bool engine_finished(ServeEngine *e) {
  if (!e->running) return true;
  const cudaError_t q = cudaEventQuery(e->ended);
  if (q == cudaErrorNotReady) return false;
  cudaGetLastError();
  e->running = false;
  uint32_t code = 0;
  if (cudaMemcpy(&code, e->exit_code, 4, cudaMemcpyDeviceToHost) == cudaSuccess)
    e->last_exit = code;
  cudaGetLastError();
  return true;
}

int engine_launch(ServeEngine *e, unsigned long long idle_ns, cudaError_t *why = nullptr) {
  // An error an earlier call on this thread left behind is not this
  // launch's: clear it, so the check below sees the launch alone (a stale
  // error read as a failed launch left a kernel running that the engine
  // did not know of, and the next kick launched another behind it).
  cudaGetLastError();
  cudaError_t ce = cudaMemsetAsync(e->exit_code, 0, 8, e->kstream);
  if (ce == cudaSuccess) {
    k_serve<true><<<e->grid, kWarpsPerBlock * 32, 0, e->kstream>>>(
        e->graphs, e->items_d, e->tail_d, e->stop_d, e->head, e->item_next, e->slot_count,
        e->slot_tiles, e->done_d, e->passed_d, e->exit_code, idle_ns);
    ce = cudaGetLastError();
  }
  if (ce != cudaSuccess) {
    if (why) *why = ce;
    cudaGetLastError();
    set_error(WETRIC_ECUDA, "resident kernel launch: %s", cudaGetErrorString(ce));
    return WETRIC_ECUDA;
  }
  WETRIC_CUDA_TRY(cudaEventRecord(e->ended, e->kstream));
  e->running = true;
  ++e->launches;
  return WETRIC_OK;
}

}  // namespace

int serve_engine_create(DeviceContext *ctx, const ServeEngineOptions &o,
                        ServeEngine **out) {
  *out = nullptr;
  std::unique_ptr<ServeEngine> e(new ServeEngine());
  e->ctx = ctx;
  e->opt = o;
  if (!e->opt.max_slots) e->opt.max_slots = 8192;
  if (!e->opt.max_items) e->opt.max_items = 1u << 20;
  // The resident kernel's stream has the device's highest priority: when it
  // is launched while the lanes' preprocessing kernels fill the SMs, its
  // blocks are placed ahead of theirs as SMs free up. (At low priority a
  // launch under load got only the few blocks the lanes left room for, and
  // those few warps then served the whole queue for tens of seconds.)
  int lo = 0, hi = 0;
  cudaDeviceGetStreamPriorityRange(&lo, &hi);
  WETRIC_CUDA_TRY(cudaStreamCreateWithPriority(&e->kstream, cudaStreamNonBlocking, hi));
  WETRIC_CUDA_TRY(cudaStreamCreateWithFlags(&e->cstream, cudaStreamNonBlocking));
  WETRIC_CUDA_TRY(cudaEventCreateWithFlags(&e->ended, cudaEventDisableTiming));
  const uint32_t S = e->opt.max_slots, I = e->opt.max_items;
  void *d = nullptr;
  WETRIC_CUDA_TRY(cudaHostAlloc(&e->items_h, I * sizeof(ServeItem), cudaHostAllocDefault));
  WETRIC_CUDA_TRY(cudaHostAlloc(&e->tail_src, I * sizeof(unsigned long long),
                                cudaHostAllocDefault));
  WETRIC_CUDA_TRY(cudaMalloc(&e->items_d, I * sizeof(ServeItem)));
  WETRIC_CUDA_TRY(cudaMalloc(&e->tail_d, 64));
  if (!(e->ctl_h = static_cast<unsigned long long *>(host_mapped(64, &d)))) {
    set_error(WETRIC_ENOMEM, "mapped host memory for the serving queue");
    return WETRIC_ENOMEM;
  }
  e->ctl_d = static_cast<unsigned long long *>(d);
  e->stop_h = reinterpret_cast<uint32_t *>(e->ctl_h + 2);
  e->stop_d = reinterpret_cast<uint32_t *>(e->ctl_d + 2);
  if (!(e->done_h = static_cast<unsigned long long *>(host_mapped(S * 8ull, &d)))) {
    set_error(WETRIC_ENOMEM, "mapped host memory for the serving queue");
    return WETRIC_ENOMEM;
  }
  e->done_d = static_cast<unsigned long long *>(d);
  if (!(e->passed_h = static_cast<uint32_t *>(host_mapped(I * 4ull, &d)))) {
    set_error(WETRIC_ENOMEM, "mapped host memory for the serving queue");
    return WETRIC_ENOMEM;
  }
  e->passed_d = static_cast<uint32_t *>(d);
  WETRIC_CUDA_TRY(cudaMalloc(&e->graphs, S * sizeof(ServeGraph)));
  WETRIC_CUDA_TRY(cudaMalloc(&e->head, 64));
  WETRIC_CUDA_TRY(cudaMalloc(&e->item_next, I * sizeof(unsigned long long)));
  WETRIC_CUDA_TRY(cudaMalloc(&e->slot_count, S * sizeof(unsigned long long)));
  WETRIC_CUDA_TRY(cudaMalloc(&e->slot_tiles, S * sizeof(unsigned long long)));
  WETRIC_CUDA_TRY(cudaMalloc(&e->exit_code, 8));  // [0] exit status, [1] quit
  int occ = 0;
  WETRIC_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &occ, k_serve<true>, kWarpsPerBlock * 32, 0));
  // Leave room on every SM for the preprocessing kernels of arriving
  // requests (their blocks need up to 256 threads x 64 registers): half
  // the blocks that fit (at least one).
  int per_sm = e->opt.blocks_per_sm ? (int)e->opt.blocks_per_sm : occ / 2;
  if (per_sm > occ) per_sm = occ;
  if (per_sm < 1) per_sm = 1;
  e->grid = ctx->sm_count * per_sm;
  WETRIC_TRY(engine_reset_space(e.get()));
  *out = e.release();
  return WETRIC_OK;
}

void serve_engine_destroy(ServeEngine *e) {
  if (!e) return;
  cudaSetDevice(e->ctx->device);
  if (e->stop_h) {
    *reinterpret_cast<volatile uint32_t *>(e->stop_h) = 1;
    std::atomic_thread_fence(std::memory_order_seq_cst);
  }
  if (e->kstream) cudaStreamSynchronize(e->kstream);
  e->active.clear();
  e->retired.clear();
  for (void *p : {(void *)e->graphs, (void *)e->head, (void *)e->item_next,
                  (void *)e->slot_count, (void *)e->slot_tiles, (void *)e->exit_code,
                  (void *)e->items_d, (void *)e->tail_d})
    if (p) cudaFree(p);
  for (void *p : {(void *)e->items_h, (void *)e->tail_src, (void *)e->ctl_h, (void *)e->done_h,
                  (void *)e->passed_h})
    if (p) cudaFreeHost(p);
  if (e->ended) cudaEventDestroy(e->ended);
  if (e->kstream) cudaStreamDestroy(e->kstream);
  if (e->cstream) cudaStreamDestroy(e->cstream);
  cudaGetLastError();
  delete e;
}

int serve_add(ServeEngine *e, std::unique_ptr<ServePlan> &plan, uint32_t *slot) {
  std::lock_guard<std::mutex> lk(e->mu);
  if (e->next_slot >= e->opt.max_slots) {
    set_error(WETRIC_EBUSY, "serving slots used up; recycle");
    return WETRIC_EBUSY;
  }
  const uint32_t s = e->next_slot;
  ServeGraph g{};
  g.rp = plan->rp32.ptr;
  g.ci = plan->csr.col_ind;
  g.n = plan->n;
  g.act_wp = plan->act_wp.ptr;
  g.act_rb = plan->act_rb.ptr;
  g.act_d = plan->act_d.ptr;
  g.K = plan->K;
  g.tile_k = plan->tile_k.ptr;
  g.tiles = plan->tiles;
  g.W = plan->W;
  g.T = plan->T;
  g.bm = plan->bm.ptr;
  g.bm_first = plan->bm_first;
  g.S = plan->S;
  if (plan->htab.ptr) {
    g.hv.rows = plan->hrows.ptr;
    g.hv.tab = plan->htab.ptr;
  }
  if (plan->ntab.ptr) {
    g.hv.nrows = plan->nrows.ptr;
    g.hv.ntab = plan->ntab.ptr;
    g.hv.nfirst = plan->nfirst;
    g.hv.ncount = plan->ncount;
  }
  WETRIC_CUDA_TRY(cudaMemcpyAsync(e->graphs + s, &g, sizeof(g), cudaMemcpyHostToDevice,
                                  e->cstream));
  WETRIC_CUDA_TRY(cudaStreamSynchronize(e->cstream));
  ++e->next_slot;
  e->active[s] = std::move(plan);
  e->pending.push_back(s);
  *slot = s;
  return WETRIC_OK;
}

int serve_publish(ServeEngine *e, uint32_t slot, uint64_t t0, uint64_t t1) {
  std::lock_guard<std::mutex> lk(e->mu);
  if (e->published >= e->opt.max_items) {
    set_error(WETRIC_EBUSY, "serving queue full; recycle");
    return WETRIC_EBUSY;
  }
  if (slot >= e->next_slot || !e->active[slot] || t1 > e->active[slot]->tiles || t0 >= t1) {
    set_error(WETRIC_EINVAL, "bad serving item");
    return WETRIC_EINVAL;
  }
  const uint64_t q = e->published;
  ServeItem &it = e->items_h[q];
  it.slot = slot;
  it.t_begin = t0;
  it.t_end = t1;
  e->tail_src[q] = q + 1;
  // the item, then the tail that covers it, in stream order
  WETRIC_CUDA_TRY(cudaMemcpyAsync(e->items_d + q, &it, sizeof(ServeItem),
                                  cudaMemcpyHostToDevice, e->cstream));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(e->tail_d, e->tail_src + q, sizeof(unsigned long long),
                                  cudaMemcpyHostToDevice, e->cstream));
  ++e->published;
  return WETRIC_OK;
}

int serve_kick(ServeEngine *e) {
  std::lock_guard<std::mutex> lk(e->mu);
  if (!engine_finished(e)) return WETRIC_OK;
  engine_free_retired(e);
  if (engine_taken(e) >= e->published) {
    // everything published was taken; a kernel is needed only if a taken
    // item's tiles are still unfinished, which cannot be once it ended
    return WETRIC_OK;
  }
  cudaError_t why = cudaSuccess;
  const int st = engine_launch(e, (unsigned long long)e->opt.idle_us * 1000ull, &why);
  if (st != WETRIC_OK) {
    ++e->launch_errors;
    e->launch_error_code = (uint32_t)why;
  }
  return st;
}

uint64_t serve_launch_errors(ServeEngine *e, uint32_t *last_code) {
  std::lock_guard<std::mutex> lk(e->mu);
  if (last_code) *last_code = e->launch_error_code;
  return e->launch_errors;
}

int serve_poll(ServeEngine *e, std::vector<std::pair<uint32_t, uint64_t>> *done) {
  std::lock_guard<std::mutex> lk(e->mu);
  done->clear();
  std::atomic_thread_fence(std::memory_order_acquire);
  size_t keep = 0;
  for (size_t i = 0; i < e->pending.size(); ++i) {
    const uint32_t s = e->pending[i];
    ServePlan *pl = e->active[s].get();
    uint64_t count = 0;
    if (pl->tiles) {
      const unsigned long long v =
          *reinterpret_cast<volatile unsigned long long *>(e->done_h + s);
      if (!v) {
        e->pending[keep++] = s;
        continue;
      }
      count = v - 1;
    }
    if (pl->core_done) {
      // the core and shell part, counted on the request's lane stream
      const cudaError_t q = cudaEventQuery(pl->core_done);
      if (q == cudaErrorNotReady) {
        e->pending[keep++] = s;
        continue;
      }
      unsigned long long c = 0;
      if (q == cudaSuccess &&
          cudaMemcpy(&c, pl->core_acc.ptr, 8, cudaMemcpyDeviceToHost) == cudaSuccess)
        count += c;
      cudaGetLastError();
    }
    done->push_back({s, count});
    e->retired_bytes += e->active[s]->bytes;
    e->retired.push_back(std::move(e->active[s]));
  }
  e->pending.resize(keep);
  engine_finished(e);
  if (!e->running) engine_free_retired(e);
  return WETRIC_OK;
}

void serve_queue_state(ServeEngine *e, uint64_t *taken, uint64_t *published) {
  std::lock_guard<std::mutex> lk(e->mu);
  *taken = engine_taken(e);
  *published = e->published;
}

int serve_recycle(ServeEngine *e) {
  std::lock_guard<std::mutex> lk(e->mu);
  if (!e->pending.empty()) {
    set_error(WETRIC_EBUSY, "a request of this sequence space is still counting");
    return WETRIC_EBUSY;
  }
  *reinterpret_cast<volatile uint32_t *>(e->stop_h) = 1;
  std::atomic_thread_fence(std::memory_order_seq_cst);
  if (e->running) {
    WETRIC_CUDA_TRY(cudaEventSynchronize(e->ended));
    engine_finished(e);
  }
  *reinterpret_cast<volatile uint32_t *>(e->stop_h) = 0;
  engine_free_retired(e);
  return engine_reset_space(e);
}

uint64_t serve_retired_bytes(ServeEngine *e) {
  std::lock_guard<std::mutex> lk(e->mu);
  return e->retired_bytes;
}

uint64_t serve_freed_bytes(ServeEngine *e) {
  std::lock_guard<std::mutex> lk(e->mu);
  return e->freed_bytes;
}

void serve_launch_info(ServeEngine *e, uint64_t *launches, uint32_t *last_exit) {
  std::lock_guard<std::mutex> lk(e->mu);
  engine_finished(e);
  *launches = e->launches;
  *last_exit = e->last_exit;
}

void serve_space_left(ServeEngine *e, uint32_t *slots, uint32_t *items) {
  std::lock_guard<std::mutex> lk(e->mu);
  *slots = e->opt.max_slots - e->next_slot;
  *items = (uint32_t)(e->opt.max_items - e->published);
}

int serve_idle_probe(DeviceContext *ctx, uint32_t idle_us, uint32_t *exit_code,
                     double *ms) {
  ServeEngineOptions o;
  o.max_slots = 4;
  o.max_items = 4;
  ServeEngine *e = nullptr;
  WETRIC_TRY(serve_engine_create(ctx, o, &e));
  std::unique_ptr<ServeEngine, void (*)(ServeEngine *)> hold(e, serve_engine_destroy);
  cudaEvent_t a = nullptr;
  WETRIC_CUDA_TRY(cudaEventCreate(&a));
  WETRIC_CUDA_TRY(cudaEventRecord(a, e->kstream));
  int st = engine_launch(e, (unsigned long long)idle_us * 1000ull);
  if (st == WETRIC_OK) {
    const cudaError_t w = cudaEventSynchronize(e->ended);
    if (w != cudaSuccess) {
      set_error(WETRIC_ECUDA, "resident kernel: %s", cudaGetErrorString(w));
      st = WETRIC_ECUDA;
    }
  }
  float f = 0;
  if (st == WETRIC_OK) {
    cudaEventElapsedTime(&f, a, e->ended);
    engine_finished(e);
    *exit_code = e->last_exit;
    *ms = f;
  }
  cudaEventDestroy(a);
  return st;
}

}  // namespace wetric
