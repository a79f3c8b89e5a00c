// preprocess.cu -- device-side graph preprocessing.
//
// The reference builds its CSR on the host: symmetrise + drop self-loops
// (tc.cu:590-621), sort (CUB or qsort, 628-647), sequential dedup + row
// histogram (649-684), then relabels by ascending degree (688-723), keeps
// each edge once toward the higher new id (740-758) and sorts every row
// (763-784). Here all of that runs on the GPU with this library's own radix
// sort:
//
//   raw pairs --canonical (min,max) key--> sort --> unique --> degrees
//     --> stable (degree, id) rank --> (rank lo, rank hi) key --> sort
//     --> oriented CSR (u64 row offsets, u32 columns)
//
// Keys pack two ids of b = bits(n-1) bits each into 2b bits, so a sort
// costs ceil(2b / 8) digit passes. Canonicalising to (min, max) before the
// first sort halves the keys compared with the reference's symmetrised
// list. The vertex order equals that of the reference's stable CUB sort
// (its -p 1 / -p 2 styles): ascending degree, ties by ascending id.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "preprocess.cuh"
#include "primitives.cuh"

namespace wetric {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;

__device__ __forceinline__ uint64_t pack_key(uint32_t lo, uint32_t hi,
                                             uint32_t b) {
  return ((uint64_t)lo << b) | (uint64_t)hi;
}

__global__ void k_max_id(const uint32_t *__restrict__ src,
                         const uint32_t *__restrict__ dst, uint64_t P,
                         uint32_t *max_id, uint32_t *any_edge) {
  uint32_t local = 0, seen = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = src[i], d = dst[i];
    if (s != d) {
      local = max(local, max(s, d));
      seen = 1;
    }
  }
  local = __reduce_max_sync(0xffffffffu, local);
  seen = __reduce_or_sync(0xffffffffu, seen);
  if ((threadIdx.x & 31) == 0) {
    if (seen) {
      atomicMax(max_id, local);
      atomicOr(any_edge, 1u);
    }
  }
}

// keys[i] = (min, max) packed, or the all-ones sentinel for a self-loop or
// an id >= n (the latter also raises *err).
__global__ void k_canon_keys(const uint32_t *__restrict__ src,
                             const uint32_t *__restrict__ dst, uint64_t P,
                             uint32_t b, uint64_t n, uint64_t sentinel,
                             uint64_t *__restrict__ keys, uint32_t *err) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t s = src[i], d = dst[i];
    uint64_t k = sentinel;
    if (s != d) {
      if ((uint64_t)s >= n || (uint64_t)d >= n) {
        atomicCAS(err, 0u, (uint32_t)kDevColumnRange);
      } else {
        k = pack_key(min(s, d), max(s, d), b);
      }
    }
    keys[i] = k;
  }
}

// Per-tile count of keys that are not the sentinel and differ from their
// predecessor (keys sorted).
__global__ void __launch_bounds__(kThreads)
    k_unique_count(const uint64_t *__restrict__ keys, uint64_t N,
                   uint64_t sentinel, uint32_t *__restrict__ tile_counts) {
  __shared__ uint32_t warp_sums[kThreads / 32];
  const uint64_t base =
      (uint64_t)blockIdx.x * kTile + (uint64_t)threadIdx.x * kItems;
  uint32_t c = 0;
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    const uint64_t i = base + j;
    if (i < N) {
      const uint64_t k = keys[i];
      c += (k != sentinel && (i == 0 || keys[i - 1] != k)) ? 1u : 0u;
    }
  }
  uint32_t total;
  prim::block_inclusive_scan<uint32_t>(c, warp_sums, &total);
  if (threadIdx.x == 0) tile_counts[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kThreads)
    k_unique_write(const uint64_t *__restrict__ keys, uint64_t N,
                   uint64_t sentinel, const uint64_t *__restrict__ tile_off,
                   uint64_t *__restrict__ out) {
  __shared__ uint32_t warp_sums[kThreads / 32];
  const uint64_t base =
      (uint64_t)blockIdx.x * kTile + (uint64_t)threadIdx.x * kItems;
  uint32_t keep_mask = 0, c = 0;
  uint64_t k[kItems];
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    const uint64_t i = base + j;
    k[j] = 0;
    if (i < N) {
      k[j] = keys[i];
      if (k[j] != sentinel && (i == 0 || keys[i - 1] != k[j])) {
        keep_mask |= 1u << j;
        ++c;
      }
    }
  }
  uint32_t total;
  const uint32_t incl = prim::block_inclusive_scan<uint32_t>(c, warp_sums, &total);
  uint64_t pos = tile_off[blockIdx.x] + (incl - c);
#pragma unroll
  for (int j = 0; j < kItems; ++j)
    if (keep_mask & (1u << j)) out[pos++] = k[j];
}

__global__ void k_degree_undirected(const uint64_t *__restrict__ ukeys,
                                    uint64_t m, uint32_t b,
                                    uint32_t *__restrict__ deg) {
  const uint64_t mask = (b >= 64) ? ~0ull : ((1ull << b) - 1);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = ukeys[i];
    atomicAdd(&deg[(uint32_t)(k >> b)], 1u);
    atomicAdd(&deg[(uint32_t)(k & mask)], 1u);
  }
}

__global__ void k_max_u32(const uint32_t *__restrict__ a, uint64_t n,
                          uint32_t *out) {
  uint32_t local = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    local = max(local, a[i]);
  local = __reduce_max_sync(0xffffffffu, local);
  if ((threadIdx.x & 31) == 0) atomicMax(out, local);
}

__global__ void k_iota(uint32_t *__restrict__ v, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    v[i] = (uint32_t)i;
}

__global__ void k_rank_from_order(const uint32_t *__restrict__ order,
                                  uint64_t n, uint32_t *__restrict__ rank) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    rank[order[i]] = (uint32_t)i;
}

__global__ void k_orient_keys(const uint64_t *ukeys, uint64_t m, uint32_t b,
                              const uint32_t *__restrict__ rank,
                              uint64_t *okeys) {
  const uint64_t mask = (1ull << b) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = ukeys[i];
    const uint32_t ra = rank[(uint32_t)(k >> b)];
    const uint32_t rb = rank[(uint32_t)(k & mask)];
    okeys[i] = pack_key(min(ra, rb), max(ra, rb), b);
  }
}

__global__ void k_both_directions(const uint64_t *__restrict__ ukeys,
                                  uint64_t m, uint32_t b,
                                  uint64_t *__restrict__ dkeys) {
  const uint64_t mask = (1ull << b) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = ukeys[i];
    const uint32_t lo = (uint32_t)(k >> b), hi = (uint32_t)(k & mask);
    dkeys[2 * i] = pack_key(lo, hi, b);
    dkeys[2 * i + 1] = pack_key(hi, lo, b);
  }
}

__global__ void k_row_histogram(const uint64_t *__restrict__ keys, uint64_t m,
                                uint32_t b, uint32_t *__restrict__ cnt) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x)
    atomicAdd(&cnt[(uint32_t)(keys[i] >> b)], 1u);
}

__global__ void k_low_bits(const uint64_t *__restrict__ keys, uint64_t m,
                           uint32_t b, uint32_t *__restrict__ col) {
  const uint64_t mask = (1ull << b) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x)
    col[i] = (uint32_t)(keys[i] & mask);
}

// Degrees of a CSR given by row offsets (the reference's num_edges of
// preprocess_vertex_t, tc.cu:694).
__global__ void k_row_lengths(const uint64_t *__restrict__ rp, uint64_t n,
                              uint32_t *__restrict__ deg) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x)
    deg[v] = (uint32_t)(rp[v + 1] - rp[v]);
}

// Orientation of a CSR as the reference's preprocess loop does it
// (tc.cu:740-758): entry (v, w) is kept as (rank v, rank w) when
// rank w > rank v. One warp per row; pass 1 counts, pass 2 writes.
__global__ void k_kept_per_row(const uint64_t *__restrict__ rp,
                               const uint32_t *__restrict__ ci, uint64_t n,
                               const uint32_t *__restrict__ rank,
                               uint32_t *__restrict__ kept) {
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t v = warp; v < n; v += nwarps) {
    const uint32_t rv = rank[v];
    uint32_t c = 0;
    for (uint64_t j = rp[v] + lane; j < rp[v + 1]; j += 32)
      c += rank[ci[j]] > rv ? 1u : 0u;
    c = __reduce_add_sync(0xffffffffu, c);
    if (lane == 0) kept[v] = c;
  }
}

__global__ void k_kept_write(const uint64_t *__restrict__ rp,
                             const uint32_t *__restrict__ ci, uint64_t n,
                             const uint32_t *__restrict__ rank, uint32_t b,
                             const uint64_t *__restrict__ off,
                             uint64_t *__restrict__ okeys) {
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  for (uint64_t v = warp; v < n; v += nwarps) {
    const uint32_t rv = rank[v];
    uint64_t pos = off[v];
    const uint64_t end = rp[v + 1];
    for (uint64_t j0 = rp[v]; j0 < end; j0 += 32) {
      const uint64_t j = j0 + lane;
      bool keep = false;
      uint32_t rw = 0;
      if (j < end) {
        rw = rank[ci[j]];
        keep = rw > rv;
      }
      const uint32_t bal = __ballot_sync(0xffffffffu, keep);
      if (keep) okeys[pos + __popc(bal & lt)] = pack_key(rv, rw, b);
      pos += __popc(bal);
    }
  }
}

// Row offsets monotone from 0 to m, every column id < n.
__global__ void k_check_ids(const uint64_t *__restrict__ rp,
                            const uint32_t *__restrict__ ci, uint64_t n,
                            uint64_t m, uint32_t *err) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x)
    if (ci[i] >= n) atomicCAS(err, 0u, (uint32_t)kDevColumnRange);
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x)
    if (rp[v + 1] < rp[v] || rp[v + 1] > m)
      atomicCAS(err, 0u, (uint32_t)kDevRowPtrRange);
  if (blockIdx.x == 0 && threadIdx.x == 0)
    if (rp[0] != 0 || rp[n] != m) atomicCAS(err, 0u, (uint32_t)kDevRowPtrRange);
}

// Grid of a grid-stride element-wise kernel: at most 32 blocks per SM, so
// blocks stay short and a higher-priority stream's kernels get SMs soon.
unsigned grid_for(DeviceContext *ctx, uint64_t work) {
  const uint64_t cap = (uint64_t)ctx->sm_count * 32;
  uint64_t g = ceil_div(work, 256);
  if (g > cap) g = cap;
  if (g == 0) g = 1;
  return (unsigned)g;
}

int read_u32(cudaStream_t st, const uint32_t *d, uint32_t *h) {
  WETRIC_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(uint32_t),
                                  cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  return WETRIC_OK;
}

int read_u64(cudaStream_t st, const uint64_t *d, uint64_t *h) {
  WETRIC_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(uint64_t),
                                  cudaMemcpyDeviceToHost, st));
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  return WETRIC_OK;
}

int dev_error(cudaStream_t st, const uint32_t *d_err, const char *what) {
  uint32_t e = 0;
  WETRIC_TRY(read_u32(st, d_err, &e));
  if (e != kDevOk) {
    set_error(WETRIC_EINVAL, "%s: invalid input (device check %u)", what, e);
    return WETRIC_EINVAL;
  }
  return WETRIC_OK;
}

// Sorted, deduplicated compaction of `keys` (sorted, with sentinel) into
// `out`; returns the number kept in *m.
int unique_sorted(DeviceContext *ctx, cudaStream_t st, const uint64_t *keys,
                  uint64_t N, uint64_t sentinel, uint64_t *out, uint64_t *m) {
  const uint64_t tiles = N == 0 ? 1 : ceil_div(N, kTile);
  Scratch<uint32_t> counts;
  Scratch<uint64_t> offs;
  WETRIC_TRY(counts.alloc(ctx, st, tiles));
  WETRIC_TRY(offs.alloc(ctx, st, tiles + 1));
  k_unique_count<<<(unsigned)tiles, kThreads, 0, st>>>(keys, N, sentinel,
                                                       counts.ptr);
  WETRIC_LAUNCH_CHECK();
  WETRIC_TRY((prim::exclusive_scan<uint32_t, uint64_t>(ctx, st, counts.ptr,
                                                       offs.ptr, tiles)));
  k_unique_write<<<(unsigned)tiles, kThreads, 0, st>>>(keys, N, sentinel,
                                                       offs.ptr, out);
  WETRIC_LAUNCH_CHECK();
  return read_u64(st, offs.ptr + tiles, m);
}

// Group of every vertex of a disjoint union: key = (group << dbits) | deg,
// group = the g with group_base[g] <= v < group_base[g + 1].
__global__ void k_group_keys(const uint32_t *__restrict__ deg, uint64_t n,
                             const uint64_t *__restrict__ group_base,
                             uint32_t G, uint32_t dbits,
                             uint64_t *__restrict__ keys) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t lo = 0, len = G;
    while (len > 1) {
      const uint32_t h = len >> 1;
      if (group_base[lo + h] <= v) lo += h;
      len -= h;
    }
    keys[v] = ((uint64_t)lo << dbits) | deg[v];
  }
}

// Within-group rank: vertices of a disjoint union ordered by (group,
// degree, id), so every group keeps its id range and the order inside a
// group is the stable ascending-degree order of that group alone.
int grouped_degree_rank(DeviceContext *ctx, cudaStream_t st,
                        const uint32_t *deg, uint64_t n,
                        const uint64_t *group_base, uint32_t G,
                        uint32_t *rank) {
  Scratch<uint64_t> k0, k1;
  Scratch<uint32_t> v0, v1, dmax;
  WETRIC_TRY(k0.alloc(ctx, st, n));
  WETRIC_TRY(k1.alloc(ctx, st, n));
  WETRIC_TRY(v0.alloc(ctx, st, n));
  WETRIC_TRY(v1.alloc(ctx, st, n));
  WETRIC_TRY(dmax.alloc(ctx, st, 1));
  WETRIC_CUDA_TRY(cudaMemsetAsync(dmax.ptr, 0, sizeof(uint32_t), st));
  k_max_u32<<<grid_for(ctx, n), 256, 0, st>>>(deg, n, dmax.ptr);
  WETRIC_LAUNCH_CHECK();
  uint32_t maxdeg = 0;
  WETRIC_TRY(read_u32(st, dmax.ptr, &maxdeg));
  const uint32_t dbits = bits_for(maxdeg);
  const uint32_t gbits = bits_for(G ? G - 1 : 0);
  k_group_keys<<<grid_for(ctx, n), 256, 0, st>>>(deg, n, group_base, G, dbits,
                                                 k0.ptr);
  WETRIC_LAUNCH_CHECK();
  k_iota<<<grid_for(ctx, n), 256, 0, st>>>(v0.ptr, n);
  WETRIC_LAUNCH_CHECK();
  bool alt = false;
  WETRIC_TRY((prim::radix_sort<uint64_t, uint32_t>(
      ctx, st, k0.ptr, k1.ptr, v0.ptr, v1.ptr, n, dbits + gbits, &alt)));
  const uint32_t *order = alt ? v1.ptr : v0.ptr;
  k_rank_from_order<<<grid_for(ctx, n), 256, 0, st>>>(order, n, rank);
  WETRIC_LAUNCH_CHECK();
  return WETRIC_OK;
}

// rank[v] = position of v in the stable ascending-degree order.
int degree_rank(DeviceContext *ctx, cudaStream_t st, const uint32_t *deg,
                uint64_t n, uint32_t *rank) {
  Scratch<uint32_t> k0, k1, v0, v1, dmax;
  WETRIC_TRY(k0.alloc(ctx, st, n));
  WETRIC_TRY(k1.alloc(ctx, st, n));
  WETRIC_TRY(v0.alloc(ctx, st, n));
  WETRIC_TRY(v1.alloc(ctx, st, n));
  WETRIC_TRY(dmax.alloc(ctx, st, 1));
  WETRIC_CUDA_TRY(cudaMemsetAsync(dmax.ptr, 0, sizeof(uint32_t), st));
  WETRIC_CUDA_TRY(cudaMemcpyAsync(k0.ptr, deg, n * sizeof(uint32_t),
                                  cudaMemcpyDeviceToDevice, st));
  k_max_u32<<<grid_for(ctx, n), 256, 0, st>>>(deg, n, dmax.ptr);
  WETRIC_LAUNCH_CHECK();
  k_iota<<<grid_for(ctx, n), 256, 0, st>>>(v0.ptr, n);
  WETRIC_LAUNCH_CHECK();
  uint32_t maxdeg = 0;
  WETRIC_TRY(read_u32(st, dmax.ptr, &maxdeg));
  bool alt = false;
  WETRIC_TRY((prim::radix_sort<uint32_t, uint32_t>(
      ctx, st, k0.ptr, k1.ptr, v0.ptr, v1.ptr, n, bits_for(maxdeg), &alt)));
  const uint32_t *order = alt ? v1.ptr : v0.ptr;
  k_rank_from_order<<<grid_for(ctx, n), 256, 0, st>>>(order, n, rank);
  WETRIC_LAUNCH_CHECK();
  return WETRIC_OK;
}

// Sorted packed (row, col) keys -> CSR arrays.
int keys_to_csr(DeviceContext *ctx, cudaStream_t st, const uint64_t *keys,
                uint64_t m, uint64_t n, uint32_t b, uint64_t *row_ptr,
                uint32_t *col_ind) {
  Scratch<uint32_t> cnt;
  WETRIC_TRY(cnt.alloc(ctx, st, n));
  WETRIC_CUDA_TRY(cudaMemsetAsync(cnt.ptr, 0, n * sizeof(uint32_t), st));
  if (m > 0) {
    k_row_histogram<<<grid_for(ctx, m), 256, 0, st>>>(keys, m, b, cnt.ptr);
    WETRIC_LAUNCH_CHECK();
    k_low_bits<<<grid_for(ctx, m), 256, 0, st>>>(keys, m, b, col_ind);
    WETRIC_LAUNCH_CHECK();
  }
  WETRIC_TRY((prim::exclusive_scan<uint32_t, uint64_t>(ctx, st, cnt.ptr,
                                                       row_ptr, n)));
  return WETRIC_OK;
}

}  // namespace

void DeviceCsr::release() {
  if (ctx) {
    if (row_ptr) dev_free(ctx, stream, row_ptr, (n + 1) * sizeof(uint64_t));
    if (col_ind) dev_free(ctx, stream, col_ind, (m ? m : 4) * sizeof(uint32_t));
  }
  row_ptr = nullptr;
  col_ind = nullptr;
  n = m = 0;
}

static int alloc_csr(DeviceContext *ctx, cudaStream_t st, uint64_t n,
                     uint64_t m, DeviceCsr *out) {
  out->release();
  out->ctx = ctx;
  out->stream = st;
  void *p = nullptr;
  WETRIC_TRY(dev_alloc(ctx, st, (n + 1) * sizeof(uint64_t), &p));
  out->row_ptr = static_cast<uint64_t *>(p);
  out->n = n;
  p = nullptr;
  int rc = dev_alloc(ctx, st, (m ? m : 4) * sizeof(uint32_t), &p);
  if (rc != WETRIC_OK) {
    out->release();
    return rc;
  }
  out->col_ind = static_cast<uint32_t *>(p);
  out->m = m;
  return WETRIC_OK;
}

// Raw pairs -> unique undirected edges as sorted canonical keys.
static int unique_edges(DeviceContext *ctx, cudaStream_t st,
                        const uint32_t *src, const uint32_t *dst, uint64_t P,
                        uint64_t n_hint, uint64_t *n_out, uint32_t *b_out,
                        Scratch<uint64_t> *ukeys, uint64_t *m_out) {
  Scratch<uint32_t> small;
  WETRIC_TRY(small.alloc(ctx, st, 4));
  WETRIC_CUDA_TRY(cudaMemsetAsync(small.ptr, 0, 4 * sizeof(uint32_t), st));
  uint64_t n = n_hint;
  if (n == 0) {
    if (P > 0) {
      k_max_id<<<grid_for(ctx, P), 256, 0, st>>>(src, dst, P, small.ptr,
                                                 small.ptr + 1);
      WETRIC_LAUNCH_CHECK();
    }
    uint32_t h[2] = {0, 0};
    WETRIC_CUDA_TRY(cudaMemcpyAsync(h, small.ptr, 2 * sizeof(uint32_t),
                                    cudaMemcpyDeviceToHost, st));
    WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
    n = (uint64_t)h[0] + 1;  // tc.cu:625, max_vertex starts at 0
  }
  if (n > (1ull << 32)) {
    set_error(WETRIC_ERANGE, "n = %llu exceeds 2^32", (unsigned long long)n);
    return WETRIC_ERANGE;
  }
  uint32_t b = bits_for(n - 1);
  if (b == 0) b = 1;
  const uint64_t sentinel = (2 * b >= 64) ? ~0ull : ((1ull << (2 * b)) - 1);
  Scratch<uint64_t> keys, alt;
  WETRIC_TRY(keys.alloc(ctx, st, P));
  WETRIC_TRY(alt.alloc(ctx, st, P));
  if (P > 0) {
    k_canon_keys<<<grid_for(ctx, P), 256, 0, st>>>(src, dst, P, b, n, sentinel,
                                                   keys.ptr, small.ptr + 2);
    WETRIC_LAUNCH_CHECK();
  }
  WETRIC_TRY(dev_error(st, small.ptr + 2, "edge ids"));
  bool in_alt = false;
  WETRIC_TRY((prim::radix_sort<uint64_t, uint32_t>(
      ctx, st, keys.ptr, alt.ptr, nullptr, nullptr, P, 2 * b, &in_alt)));
  uint64_t *sorted = in_alt ? alt.ptr : keys.ptr;
  uint64_t *spare = in_alt ? keys.ptr : alt.ptr;
  uint64_t m = 0;
  WETRIC_TRY(unique_sorted(ctx, st, sorted, P, sentinel, spare, &m));
  // Keep the buffer that holds the unique keys; release the other.
  if (in_alt) {
    alt.release();
    ukeys->ctx = keys.ctx;
    ukeys->stream = keys.stream;
    ukeys->bytes = keys.bytes;
    ukeys->ptr = keys.detach();
  } else {
    keys.release();
    ukeys->ctx = alt.ctx;
    ukeys->stream = alt.stream;
    ukeys->bytes = alt.bytes;
    ukeys->ptr = alt.detach();
  }
  *n_out = n;
  *b_out = b;
  *m_out = m;
  return WETRIC_OK;
}

int orient_pairs(DeviceContext *ctx, cudaStream_t st, const uint32_t *src,
                 const uint32_t *dst, uint64_t P, uint64_t n_hint,
                 DeviceCsr *out, const uint64_t *group_base, uint32_t G) {
  NvtxRange nvtx_("wetric orient");
  uint64_t n = 0, m = 0;
  uint32_t b = 0;
  Scratch<uint64_t> ukeys;
  WETRIC_TRY(unique_edges(ctx, st, src, dst, P, n_hint, &n, &b, &ukeys, &m));
  Scratch<uint32_t> deg, rank;
  WETRIC_TRY(deg.alloc(ctx, st, n));
  WETRIC_TRY(rank.alloc(ctx, st, n));
  WETRIC_CUDA_TRY(cudaMemsetAsync(deg.ptr, 0, n * sizeof(uint32_t), st));
  if (m > 0) {
    k_degree_undirected<<<grid_for(ctx, m), 256, 0, st>>>(ukeys.ptr, m, b,
                                                          deg.ptr);
    WETRIC_LAUNCH_CHECK();
  }
  if (group_base != nullptr && G > 1) {
    WETRIC_TRY(grouped_degree_rank(ctx, st, deg.ptr, n, group_base, G, rank.ptr));
  } else {
    WETRIC_TRY(degree_rank(ctx, st, deg.ptr, n, rank.ptr));
  }
  deg.release();
  // Orientation rewrites each unique key in place (element i reads and
  // writes only position i), so only the sort's second buffer is new: the
  // peak stays at input pairs + 2 key buffers (m > 2^32 fits 180 GB).
  if (m > 0) {
    k_orient_keys<<<grid_for(ctx, m), 256, 0, st>>>(ukeys.ptr, m, b, rank.ptr,
                                                    ukeys.ptr);
    WETRIC_LAUNCH_CHECK();
  }
  rank.release();
  Scratch<uint64_t> oalt;
  WETRIC_TRY(oalt.alloc(ctx, st, m));
  bool in_alt = false;
  WETRIC_TRY((prim::radix_sort<uint64_t, uint32_t>(
      ctx, st, ukeys.ptr, oalt.ptr, nullptr, nullptr, m, 2 * b, &in_alt)));
  const uint64_t *sorted = in_alt ? oalt.ptr : ukeys.ptr;
  WETRIC_TRY(alloc_csr(ctx, st, n, m, out));
  WETRIC_TRY(keys_to_csr(ctx, st, sorted, m, n, b, out->row_ptr, out->col_ind));
  return WETRIC_OK;
}

int symmetric_from_pairs(DeviceContext *ctx, cudaStream_t st,
                         const uint32_t *src, const uint32_t *dst, uint64_t P,
                         uint64_t n_hint, DeviceCsr *out) {
  uint64_t n = 0, m = 0;
  uint32_t b = 0;
  Scratch<uint64_t> ukeys;
  WETRIC_TRY(unique_edges(ctx, st, src, dst, P, n_hint, &n, &b, &ukeys, &m));
  Scratch<uint64_t> dkeys, dalt;
  WETRIC_TRY(dkeys.alloc(ctx, st, 2 * m));
  WETRIC_TRY(dalt.alloc(ctx, st, 2 * m));
  if (m > 0) {
    k_both_directions<<<grid_for(ctx, m), 256, 0, st>>>(ukeys.ptr, m, b,
                                                        dkeys.ptr);
    WETRIC_LAUNCH_CHECK();
  }
  ukeys.release();
  bool in_alt = false;
  WETRIC_TRY((prim::radix_sort<uint64_t, uint32_t>(
      ctx, st, dkeys.ptr, dalt.ptr, nullptr, nullptr, 2 * m, 2 * b, &in_alt)));
  const uint64_t *sorted = in_alt ? dalt.ptr : dkeys.ptr;
  WETRIC_TRY(alloc_csr(ctx, st, n, 2 * m, out));
  WETRIC_TRY(
      keys_to_csr(ctx, st, sorted, 2 * m, n, b, out->row_ptr, out->col_ind));
  return WETRIC_OK;
}

int orient_csr(DeviceContext *ctx, cudaStream_t st, const uint64_t *rp,
               const uint32_t *ci, uint64_t n, uint64_t m, DeviceCsr *out) {
  if (n == 0) {
    WETRIC_TRY(alloc_csr(ctx, st, 0, 0, out));
    WETRIC_CUDA_TRY(cudaMemsetAsync(out->row_ptr, 0, sizeof(uint64_t), st));
    return WETRIC_OK;
  }
  if (n > (1ull << 32)) {
    set_error(WETRIC_ERANGE, "n = %llu exceeds 2^32", (unsigned long long)n);
    return WETRIC_ERANGE;
  }
  Scratch<uint32_t> err;
  WETRIC_TRY(err.alloc(ctx, st, 1));
  WETRIC_CUDA_TRY(cudaMemsetAsync(err.ptr, 0, sizeof(uint32_t), st));
  k_check_ids<<<grid_for(ctx, m > n ? m : n), 256, 0, st>>>(rp, ci, n, m,
                                                           err.ptr);
  WETRIC_LAUNCH_CHECK();
  WETRIC_TRY(dev_error(st, err.ptr, "csr"));
  uint32_t b = bits_for(n - 1);
  if (b == 0) b = 1;
  Scratch<uint32_t> deg, rank;
  WETRIC_TRY(deg.alloc(ctx, st, n));
  WETRIC_TRY(rank.alloc(ctx, st, n));
  k_row_lengths<<<grid_for(ctx, n), 256, 0, st>>>(rp, n, deg.ptr);
  WETRIC_LAUNCH_CHECK();
  WETRIC_TRY(degree_rank(ctx, st, deg.ptr, n, rank.ptr));
  // deg is reused as the per-row kept count.
  const unsigned warps_grid = grid_for(ctx, n * 32);
  k_kept_per_row<<<warps_grid, 256, 0, st>>>(rp, ci, n, rank.ptr, deg.ptr);
  WETRIC_LAUNCH_CHECK();
  Scratch<uint64_t> off;
  WETRIC_TRY(off.alloc(ctx, st, n + 1));
  WETRIC_TRY((prim::exclusive_scan<uint32_t, uint64_t>(ctx, st, deg.ptr,
                                                       off.ptr, n)));
  uint64_t kept = 0;
  WETRIC_TRY(read_u64(st, off.ptr + n, &kept));
  Scratch<uint64_t> okeys, oalt;
  WETRIC_TRY(okeys.alloc(ctx, st, kept));
  WETRIC_TRY(oalt.alloc(ctx, st, kept));
  k_kept_write<<<warps_grid, 256, 0, st>>>(rp, ci, n, rank.ptr, b, off.ptr,
                                           okeys.ptr);
  WETRIC_LAUNCH_CHECK();
  deg.release();
  rank.release();
  off.release();
  bool in_alt = false;
  WETRIC_TRY((prim::radix_sort<uint64_t, uint32_t>(
      ctx, st, okeys.ptr, oalt.ptr, nullptr, nullptr, kept, 2 * b, &in_alt)));
  const uint64_t *sorted = in_alt ? oalt.ptr : okeys.ptr;
  WETRIC_TRY(alloc_csr(ctx, st, n, kept, out));
  WETRIC_TRY(
      keys_to_csr(ctx, st, sorted, kept, n, b, out->row_ptr, out->col_ind));
  return WETRIC_OK;
}

}  // namespace wetric
