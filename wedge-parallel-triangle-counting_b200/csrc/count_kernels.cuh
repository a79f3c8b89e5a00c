// count_kernels.cuh -- device code of the wedge count, shared by the
// single-graph path (count.cu) and the batched path (batch.cu). Everything is
// in an unnamed namespace: each translation unit instantiates what it uses.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace wetric {
namespace {

constexpr uint32_t kDefaultBlock = 256;
constexpr uint32_t kKernelBlockTile = 1;
constexpr uint64_t kMaxOutDegree = 1ull << 30;  // integer decode limit

template <typename Off>
__device__ __forceinline__ uint64_t ld_off(const Off *p, uint64_t i) {
  return (uint64_t)__ldg(p + i);
}

// Bitmap words are loaded with an L2 evict-last cache policy: the bitmap (a
// few MB) then outlasts the streaming hash-bucket lines in L2, and the L2
// requests marked evict-last are exactly the bitmap's loads, so a profiler
// reads the bitmap's own L2 hit rate from them
// (lts__t_requests_evict_last_lookup_hit / lts__t_requests_evict_last).
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
  uint64_t pol;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ uint32_t ld_bitmap(const uint32_t *p, uint64_t pol) {
  uint32_t v;
  asm("ld.global.nc.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}

// floor(sqrt(x)) for x < 2^62. The float (x < 2^48) or double estimate
// is within 2 of the answer there, so two bounded correction steps each way
// suffice; no loop depends on the data.
__device__ __forceinline__ uint64_t isqrt64(uint64_t x) {
  uint64_t y;
  if (x < (1ull << 48)) {
    y = (uint64_t)__fsqrt_rn((float)x);
  } else {
    y = (uint64_t)__dsqrt_rn((double)x);
  }
  if (y > 0xFFFFFFFFull) y = 0xFFFFFFFFull;
#pragma unroll
  for (int k = 0; k < 2; ++k) y -= (y * y > x) ? 1 : 0;
#pragma unroll
  for (int k = 0; k < 2; ++k) y += ((y + 1) * (y + 1) <= x) ? 1 : 0;
  return y;
}

// Wedge iv (0-based) of a vertex with out-degree d, in row-major order of
// the strict upper triangle: returns (wi, ui), wi < ui < d. Counting rows
// from the end, the last q rows hold q(q+1)/2 wedges, so with
// j = C(d,2) - 1 - iv the row from the end is q = (isqrt(8j+1) - 1) / 2.
// Same mapping as the floating-point formula of tc.cu:211-212, without
// floating-point rounding.
// Returns false (and no indices) when iv is not a wedge of the vertex, so
// a caller's indexing mistake can never turn into an out-of-row load.
// Vertices with d < 2^16 (every vertex of most graphs) take a 32-bit path:
// j < 2^31, x = 8j + 1 < 2^34, and the single-instruction approximate
// square root of the float x is within 0.1 of sqrt(x) there (float rounding
// of x: relative 2^-23; sqrt.approx.f32: relative error below 2^-22; times
// sqrt(x) < 2^17), so one correction step each way gives floor(sqrt(x)).
__device__ __forceinline__ uint32_t isqrt_small(uint32_t j) {
  const float f = __fmaf_rn(8.0f, __uint2float_rn(j), 1.0f);
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(f));
  uint32_t y = __float2uint_rz(r);
  const uint64_t x = 8ull * j + 1;
  y -= ((uint64_t)y * y > x) ? 1u : 0u;
  y += ((uint64_t)(y + 1) * (y + 1) <= x) ? 1u : 0u;
  return y;
}

__device__ __forceinline__ bool decode_wedge(uint64_t iv, uint64_t d,
                                             uint32_t *wi, uint32_t *ui) {
  if (d < 65536) {
    const uint32_t d32 = (uint32_t)d;
    const uint32_t W32 = d32 * (d32 - 1) / 2;  // < 2^31
    if (d32 < 2 || iv >= W32) return false;
    const uint32_t j = W32 - 1 - (uint32_t)iv;
    const uint32_t q = (isqrt_small(j) - 1) >> 1;
    const uint32_t p = j - q * (q + 1) / 2;
    if (q > d32 - 2 || p > q) return false;
    *wi = d32 - 2 - q;
    *ui = d32 - 1 - p;
    return true;
  }
  const uint64_t W = d * (d - 1) / 2;
  if (iv >= W) return false;
  const uint64_t j = W - 1 - iv;
  const uint64_t q = (isqrt64(8 * j + 1) - 1) >> 1;
  const uint64_t p = j - q * (q + 1) / 2;
  if (q > d - 2 || p > q) return false;
  *wi = (uint32_t)(d - 2 - q);
  *ui = (uint32_t)(d - 1 - p);
  return true;
}

template <typename Off>
__global__ void k_vertex_wedges(const Off *__restrict__ rp, uint64_t n,
                                uint64_t m, uint32_t *__restrict__ active,
                                unsigned long long *__restrict__ maxdeg,
                                uint32_t *err) {
  uint64_t local_max = 0;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = ld_off(rp, v), e = ld_off(rp, v + 1);
    if (e < b || e > m) {
      atomicCAS(err, 0u, (uint32_t)kDevRowPtrRange);
      active[v] = 0;
      continue;
    }
    const uint64_t d = e - b;
    active[v] = d >= 2 ? 1u : 0u;
    local_max = max(local_max, d);
  }
  for (int o = 16; o > 0; o >>= 1)
    local_max = max(local_max, __shfl_down_sync(0xffffffffu, local_max, o));
  if ((threadIdx.x & 31) == 0) atomicMax(maxdeg, (unsigned long long)local_max);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (ld_off(rp, 0) != 0 || ld_off(rp, n) != m)
      atomicCAS(err, 0u, (uint32_t)kDevRowPtrRange);
  }
}

template <typename Off>
__global__ void k_compact_active(const Off *__restrict__ rp, uint64_t n,
                                 const uint32_t *__restrict__ active,
                                 const uint64_t *__restrict__ pos,
                                 uint64_t *__restrict__ act_wc,
                                 uint64_t *__restrict__ act_rb,
                                 uint32_t *__restrict__ act_d) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    if (active[v]) {
      const uint64_t k = pos[v];
      const uint64_t b = ld_off(rp, v), d = ld_off(rp, v + 1) - b;
      act_wc[k] = d * (d - 1) / 2;
      act_rb[k] = b;
      act_d[k] = (uint32_t)d;
    }
  }
}

// Wedge prefix at given vertices: out[i] = number of wedges of the
// vertices below rows.v[i] (act_wp over the active vertices, pos the
// active-vertex index of every vertex, both with an entry for n).
struct ChunkRows {
  uint64_t v[kMaxColChunks];
  uint32_t c;
};
__global__ void k_chunk_prefix(const uint64_t *__restrict__ act_wp,
                               const uint64_t *__restrict__ pos, ChunkRows rows,
                               uint64_t *__restrict__ out) {
  const uint32_t i = threadIdx.x;
  if (i < rows.c) out[i] = act_wp[pos[rows.v[i]]];
}

// tile_k[t] = largest k with act_wp[k] <= (wb + t*T), t in [0, tiles);
// tile_k[tiles] = the same for wedge we-1.
__global__ void k_tile_map(const uint64_t *__restrict__ act_wp, uint64_t K,
                           uint64_t wb, uint64_t we, uint64_t T,
                           uint64_t tiles, uint32_t *__restrict__ tile_k) {
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
       t <= tiles; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = t < tiles ? wb + t * T : we - 1;
    uint64_t lo = 0, len = K;
    while (len > 1) {
      const uint64_t h = len >> 1;
      if (act_wp[lo + h] <= i) lo += h;
      len -= h;
    }
    tile_k[t] = (uint32_t)lo;
  }
}

// One warp per bitmap row v in [n - min(n, a), n): sets bit
// S - (n-v)(n-v-1)/2 + w - v - 1 for every out-neighbour w (tc.cu:334-346).
// Rows [first_row, row_end) of the bitmap (row_end <= n: a part of it).
template <typename Off>
__global__ void k_bitmap(const Off *__restrict__ rp,
                         const uint32_t *__restrict__ ci, uint64_t n,
                         uint64_t first_row, uint64_t S,
                         uint32_t *__restrict__ bm, uint64_t row_end = ~0ull) {
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t end = row_end < n ? row_end : n;
  for (uint64_t v = first_row + warp; v < end; v += nwarps) {
    const uint64_t base = S - (n - v) * (n - v - 1) / 2;
    const uint64_t e = ld_off(rp, v + 1);
    for (uint64_t j = ld_off(rp, v) + lane; j < e; j += 32) {
      const uint64_t w = ci[j];
      if (w > v && w < n) {
        const uint64_t idx = base + w - v - 1;
        if (idx < S) atomicOr(&bm[idx >> 5], 1u << (idx & 31));
      }
    }
  }
}

// Rows sorted strictly ascending, every column > row and < n.
// Rows with broken offsets are skipped here (k_vertex_wedges reports them).
template <typename Off>
__global__ void k_validate(const Off *__restrict__ rp,
                           const uint32_t *__restrict__ ci, uint64_t n,
                           uint64_t m, uint32_t *err) {
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t v = warp; v < n; v += nwarps) {
    const uint64_t b = ld_off(rp, v), e = ld_off(rp, v + 1);
    if (e < b || e > m) continue;
    for (uint64_t j = b + lane; j < e; j += 32) {
      const uint64_t c = ci[j];
      if (c >= n) atomicCAS(err, 0u, (uint32_t)kDevColumnRange);
      else if (c <= v) atomicCAS(err, 0u, (uint32_t)kDevNotOriented);
      else if (j > b && ci[j - 1] >= c) atomicCAS(err, 0u, (uint32_t)kDevUnsortedRow);
    }
  }
}

template <typename Off>
__global__ void k_count(const Off *__restrict__ rp,
                        const uint32_t *__restrict__ ci, uint64_t n,
                        const uint64_t *__restrict__ act_wp,
                        const uint64_t *__restrict__ act_rb,
                        const uint32_t *__restrict__ act_d,
                        const uint32_t *__restrict__ tile_k, uint64_t tiles,
                        uint64_t wb, uint64_t we, uint32_t s,
                        const uint32_t *__restrict__ bm, uint64_t bm_first,
                        uint64_t S, unsigned long long *__restrict__ out) {
  extern __shared__ uint64_t s_wp[];  // T + 1 entries
  __shared__ unsigned long long warp_acc[32];
  const uint32_t B = blockDim.x;
  const uint64_t T = (uint64_t)B * s;
  uint64_t acc = 0;
  for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const uint64_t i0 = wb + t * T;
    const uint32_t klo = tile_k[t];
    const uint32_t span = tile_k[t + 1] - klo + 1;
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < span; j += B) s_wp[j] = act_wp[klo + j];
    __syncthreads();
    uint32_t c = 0;
    for (uint32_t r = 0; r < s; ++r) {
      const uint64_t i = i0 + (uint64_t)r * B + threadIdx.x;
      if (i >= we) break;
      uint32_t lo = 0, len = span;
      while (len > 1) {
        const uint32_t h = len >> 1;
        if (s_wp[lo + h] <= i) lo += h;
        len -= h;
      }
      const uint64_t k = (uint64_t)klo + lo;
      const uint64_t iv = i - s_wp[lo];
      const uint64_t rb = __ldg(act_rb + k);
      const uint64_t d = __ldg(act_d + k);
      uint32_t wi, ui;
      if (!decode_wedge(iv, d, &wi, &ui)) continue;
      const uint32_t w = __ldg(ci + rb + wi);
      const uint32_t u = __ldg(ci + rb + ui);
      uint32_t hit = 0;
      if ((uint64_t)w >= bm_first) {
        if (u > w && (uint64_t)u < n) {
          const uint64_t nw = n - w;
          const uint64_t idx = S - nw * (nw - 1) / 2 + (u - w - 1);
          if (idx < S) hit = (__ldg(bm + (idx >> 5)) >> (idx & 31)) & 1u;
        }
      } else if ((uint64_t)w < n) {
        const uint64_t b = ld_off(rp, w);
        uint64_t len2 = ld_off(rp, w + 1) - b;
        if (len2 > 0) {
          const uint32_t *p = ci + b;
          while (len2 > 1) {
            const uint64_t h = len2 >> 1;
            p = (__ldg(p + h) <= u) ? p + h : p;
            len2 -= h;
          }
          hit = (__ldg(p) == u) ? 1u : 0u;
        }
      }
      c += hit;
    }
    acc += c;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) warp_acc[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long tot = 0;
    for (uint32_t w = 0; w < (B >> 5); ++w) tot += warp_acc[w];
    if (tot) atomicAdd(out, tot);
  }
}

// Warp-staged count. Each warp takes whole tiles of G = 256 * s
// consecutive wedges from a global counter and walks them in rounds of 32
// (lane l takes wedge base + l):
//   * vertex lookup: the round's 32 wedges belong to at most 32 consecutive
//     active vertices starting at the warp's current vertex, so one
//     coalesced load of 32 prefix / row-start / degree entries and a 5-step
//     shuffle search give every lane its vertex;
//   * edge check: lanes whose middle vertex w is in the bitmap test one bit;
//     for the others the warp stages N+(w) of its last searching lane in
//     shared memory (coalesced loads, reused while later rounds stay on the
//     same row) and those lanes binary-search on chip; the remaining lanes
//     (another row in a round that straddles two, or d+(w) > kStageCap)
//     search global memory.
constexpr int kStageCap = 1024;
constexpr int kWarpsPerBlock = 8;

// Per-graph view of a batch (a disjoint union of graphs, each owning a
// contiguous id range and a contiguous wedge range). Unused (all null) for
// a single graph.
struct BatchView {
  uint32_t G;                // graphs
  const uint64_t *tile_prefix;  // [G+1] first tile of each graph
  const uint32_t *tile_size;    // [G] wedges per tile of each graph
  const uint64_t *wbase;        // [G+1] first wedge of each graph
  const uint32_t *act_g;     // graph of each active vertex
  const uint64_t *vbase;     // [G+1] first id of each graph
  const uint64_t *bm_first;  // [G] first local id in the graph's bitmap
                             //     (== n_g when the graph has no bitmap)
  const uint64_t *bm_S;      // [G] bits of the graph's bitmap, a_g(a_g-1)/2
  const uint64_t *bm_off;    // [G] first word of the graph's bitmap
  // [G x 8] u32, 32-byte records read with one load by the count: first
  // id, n_g, bitmap first local id, bitmap first word (lo, hi), bitmap
  // bits S_g (lo, hi), 0.
  const uint32_t *ginfo;
  unsigned long long *counts;  // [G] per-graph triangles (output)
};

// Wedge range [*base, *end) of tile t: uniform tiles of G wedges from wb
// for one graph; for a batch, tile t belongs to the graph g with
// tile_prefix[g] <= t < tile_prefix[g+1] and graph g's tiles have
// tile_size[g] wedges each, starting at wbase[g].
template <bool kBatch>
__device__ __forceinline__ void tile_bounds(uint64_t t, uint64_t wb,
                                            uint64_t we, uint64_t G,
                                            const BatchView &bv,
                                            uint64_t *base, uint64_t *end) {
  if (kBatch) {
    uint32_t lo = 0, len = bv.G;
    while (len > 1) {
      const uint32_t h = len >> 1;
      if (__ldg(bv.tile_prefix + lo + h) <= t) lo += h;
      len -= h;
    }
    const uint64_t T = __ldg(bv.tile_size + lo);
    *base = __ldg(bv.wbase + lo) + (t - __ldg(bv.tile_prefix + lo)) * T;
    *end = min(*base + T, __ldg(bv.wbase + lo + 1));
  } else {
    *base = wb + t * G;
    *end = min(*base + G, we);
  }
}

// Batch tile map: tile_k[t] = active vertex owning the first wedge of
// tile t (tile t's range as in tile_bounds<true>).
__global__ void k_batch_tile_map(const uint64_t *__restrict__ act_wp,
                                 uint64_t K, uint64_t tiles, BatchView bv,
                                 uint32_t *__restrict__ tile_k) {
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < tiles;
       t += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t base, end;
    tile_bounds<true>(t, 0, 0, 0, bv, &base, &end);
    uint64_t lo = 0, len = K;
    while (len > 1) {
      const uint64_t h = len >> 1;
      if (act_wp[lo + h] <= base) lo += h;
      len -= h;
    }
    tile_k[t] = (uint32_t)lo;
  }
}

// Warp sum of c, added by lane 0 to *dst (c reset by the caller).
__device__ __forceinline__ void flush_count(uint32_t c,
                                            unsigned long long *dst) {
  const uint32_t tot = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0 && tot && dst) atomicAdd(dst, (unsigned long long)tot);
}

template <typename Off, bool kBatch>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    k_count_staged(const Off *__restrict__ rp, const uint32_t *__restrict__ ci,
                   uint64_t n, const uint64_t *__restrict__ act_wp,
                   const uint64_t *__restrict__ act_rb,
                   const uint32_t *__restrict__ act_d, uint64_t K,
                   const uint32_t *__restrict__ tile_k, uint64_t tiles,
                   uint64_t wb, uint64_t we, uint64_t G,
                   const uint32_t *__restrict__ bm, uint64_t bm_first,
                   uint64_t S, unsigned long long *__restrict__ next_tile,
                   unsigned long long *__restrict__ out, BatchView bv) {
  __shared__ uint32_t stage[kWarpsPerBlock][kStageCap];
  __shared__ unsigned long long warp_acc[kWarpsPerBlock];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t *buf = stage[warp];
  uint64_t staged = ~0ull;  // vertex whose row is in buf (warp-uniform)
  uint32_t staged_d = 0;
  uint64_t acc = 0;
  uint32_t cur_g = 0xFFFFFFFFu;  // batch: graph of the pending count c
  for (;;) {
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(next_tile, 1ull);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= tiles) break;
    uint64_t base, end;
    tile_bounds<kBatch>(t, wb, we, G, bv, &base, &end);
    uint64_t kcur = tile_k[t];
    uint32_t c = 0;
    for (; base < end; base += 32) {
      const uint64_t i = base + lane;
      const bool valid = i < end;
      // 32-entry vertex window starting at kcur.
      const uint64_t kl = kcur + lane;
      const uint64_t E = kl <= K ? __ldg(act_wp + kl) : ~0ull;
      const uint64_t RB = kl < K ? __ldg(act_rb + kl) : 0;
      const uint32_t D = kl < K ? __ldg(act_d + kl) : 2u;
      uint32_t GW = 0;
      if (kBatch) GW = kl < K ? __ldg(bv.act_g + kl) : 0u;
      uint32_t j = 0;
#pragma unroll
      for (uint32_t step = 16; step > 0; step >>= 1) {
        const uint64_t e = __shfl_sync(0xffffffffu, E, j + step);
        if (e <= i) j += step;
      }
      const uint64_t e0 = __shfl_sync(0xffffffffu, E, j);
      const uint64_t rb = __shfl_sync(0xffffffffu, RB, j);
      const uint64_t d = __shfl_sync(0xffffffffu, D, j);
      const uint32_t g = kBatch ? __shfl_sync(0xffffffffu, GW, j) : 0u;
      // Next round starts at wedge base + 32: on the vertex of this round's
      // last wedge (kcur + j31), or on the next one when that vertex ends
      // exactly at base + 32 (its successor's prefix, entry j31 + 1, which
      // is entry 32 -- one past the window -- when j31 == 31).
      {
        const uint32_t j31 = __shfl_sync(0xffffffffu, j, 31);
        const uint64_t k32 = kcur + 32;
        const uint64_t E32 = k32 <= K ? __ldg(act_wp + k32) : ~0ull;
        const uint64_t e_next =
            j31 < 31 ? __shfl_sync(0xffffffffu, E, (j31 + 1) & 31) : E32;
        kcur += j31 + (e_next <= base + 32 ? 1u : 0u);
      }
      bool ok = valid;
      uint32_t w = 0, u = 0;
      if (valid) {
        uint32_t wi = 0, ui = 0;
        ok = decode_wedge(i - e0, d, &wi, &ui) && e0 <= i;
        if (ok) {
          w = __ldg(ci + rb + wi);
          u = __ldg(ci + rb + ui);
        }
      }
      bool is_bm;
      uint32_t hit = 0;
      if (kBatch) {
        // Bitmap of graph g over its own local ids.
        const uint64_t vb = ok ? __ldg(bv.vbase + g) : 0;
        const uint64_t ng = ok ? __ldg(bv.vbase + g + 1) - vb : 0;
        const uint64_t wl = (uint64_t)w - vb, ul = (uint64_t)u - vb;
        is_bm = ok && w >= vb && wl < ng && wl >= __ldg(bv.bm_first + g);
        if (is_bm && u > w && ul < ng) {
          const uint64_t Sg = __ldg(bv.bm_S + g);
          const uint64_t nw = ng - wl;
          const uint64_t idx = Sg - nw * (nw - 1) / 2 + (ul - wl - 1);
          if (idx < Sg)
            hit = (__ldg(bm + __ldg(bv.bm_off + g) + (idx >> 5)) >> (idx & 31)) & 1u;
        }
      } else {
        is_bm = ok && (uint64_t)w >= bm_first;
        if (is_bm && u > w && (uint64_t)u < n) {
          const uint64_t nw = n - w;
          const uint64_t idx = S - nw * (nw - 1) / 2 + (u - w - 1);
          if (idx < S) hit = (__ldg(bm + (idx >> 5)) >> (idx & 31)) & 1u;
        }
      }
      const bool is_srch = ok && !is_bm && (uint64_t)w < n;
      const uint32_t smask = __ballot_sync(0xffffffffu, is_srch);
      if (smask) {
        const int src = 31 - __clz(smask);
        const uint32_t wc = __shfl_sync(0xffffffffu, w, src);
        if ((uint64_t)wc != staged) {
          const uint64_t bw = ld_off(rp, wc);
          const uint64_t dw = ld_off(rp, wc + 1) - bw;
          if (dw <= (uint64_t)kStageCap) {
            __syncwarp();
            for (uint32_t q = lane; q < dw; q += 32) buf[q] = __ldg(ci + bw + q);
            __syncwarp();
            staged = wc;
            staged_d = (uint32_t)dw;
          }
        }
        if (is_srch) {
          if ((uint64_t)w == staged) {
            uint32_t len = staged_d;
            if (len > 0) {
              uint32_t p = 0;
              while (len > 1) {
                const uint32_t h = len >> 1;
                p = (buf[p + h] <= u) ? p + h : p;
                len -= h;
              }
              hit = buf[p] == u ? 1u : 0u;
            }
          } else {
            const uint64_t b = ld_off(rp, w);
            uint64_t len = ld_off(rp, w + 1) - b;
            if (len > 0) {
              const uint32_t *p = ci + b;
              while (len > 1) {
                const uint64_t h = len >> 1;
                p = (__ldg(p + h) <= u) ? p + h : p;
                len -= h;
              }
              hit = (__ldg(p) == u) ? 1u : 0u;
            }
          }
        }
      }
      if (kBatch) {
        // Per-graph accumulation: the pending count c belongs to cur_g; a
        // round that stays on cur_g adds to it, otherwise it is flushed.
        const uint32_t g0 = __shfl_sync(0xffffffffu, g, 0);
        const bool uni = __all_sync(0xffffffffu, !ok || g == g0);
        if (!(uni && g0 == cur_g)) {
          flush_count(c, cur_g != 0xFFFFFFFFu ? bv.counts + cur_g : nullptr);
          acc += c;
          c = 0;
          cur_g = 0xFFFFFFFFu;
          if (uni) {
            cur_g = g0;
          } else {
            const uint32_t key = ok ? g : 0xFFFFFFFFu;
            const uint32_t peers = __match_any_sync(0xffffffffu, key);
            const uint32_t hits = __ballot_sync(0xffffffffu, hit) & peers;
            if (ok && lane == __ffs(peers) - 1 && hits) {
              atomicAdd(bv.counts + g, (unsigned long long)__popc(hits));
            }
            acc += hit;
            hit = 0;
          }
        }
      }
      c += hit;
    }
    if (kBatch) {
      flush_count(c, cur_g != 0xFFFFFFFFu ? bv.counts + cur_g : nullptr);
      cur_g = 0xFFFFFFFFu;
    }
    acc += c;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) warp_acc[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long tot = 0;
    for (int q = 0; q < kWarpsPerBlock; ++q) tot += warp_acc[q];
    if (tot) atomicAdd(out, tot);
  }
}

// Per-row hash sets: an alternative edge-existence structure for rows too
// long for a cheap search. Row w with d+(w) >= min_degree owns
// hoff[w+1] - hoff[w] = ceil(d+(w) / keys_per_bucket) buckets of
// kHashBucket u32 slots (32 bytes, one sector) in `tab`. Column x goes to
// bucket umulhi(x * 2654435761, buckets) -- the multiplicative hash scaled
// to any bucket count -- or, when that bucket is full, the next one
// (wrapping). Slots of a bucket fill in order, so one 32-byte load
// (ld.global.nc.v8) almost always settles a lookup: found, or an empty slot
// proves absence.
constexpr uint32_t kHashBucket = 8;
constexpr uint32_t kHashMinDegree = 16;      // single-graph count
constexpr uint32_t kHashKeysPerBucket = 3;   // single-graph count
constexpr uint32_t kHashEmpty = 0xFFFFFFFFu;
constexpr uint32_t kHashMul = 2654435761u;

struct HashView {
  const uint2 *rows;    // [n] {first bucket, buckets} of each row (null: no sets)
  const uint32_t *tab;  // buckets * kHashBucket slots, 32-byte aligned
  // Near sets (kNear): rows w in [nfirst, nfirst + ncount), all with
  // n - w <= kNearSpan, keep u - w - 1 as 16-bit keys in 16-byte buckets
  // of kNearSlots slots; nrows[w - nfirst] = {first bucket, buckets}.
  const uint2 *nrows = nullptr;
  const uint32_t *ntab = nullptr;  // buckets * kNearWords words, aligned
  uint32_t nfirst = 0, ncount = 0;
};

// Near sets. For a row w with n - w <= 65536 every valid key u - w - 1 is
// at most 65534, so 16 bits hold it and 0xFFFF marks an empty slot; 8 keys
// fit one 16-byte bucket, half the bytes of the 32-bit sets per column.
// These rows are the hash rows nearest the bitmap -- the highest-degree
// ones outside it, probed most often -- so halving their sets keeps more of
// them in L2. A bucket's four words are compared at once: with
// y = word ^ (key * 0x10001), a 16-bit half of y is zero iff
// (y - 0x10001) & ~y & 0x80008000 is non-zero.
constexpr uint32_t kNearSpan = 65536;
constexpr uint32_t kNearWords = 4;               // words per near bucket
constexpr uint32_t kNearSlots = 2 * kNearWords;  // 16-bit slots per bucket
constexpr uint32_t kNearKeysPerBucket = 3;
constexpr uint32_t kNearEmpty = 0xFFFFu;
struct NearBucket {
  uint32_t w[kNearWords];
};
__device__ __forceinline__ NearBucket ld_bucket16(const uint32_t *p) {
  NearBucket b;
  if (kNearWords == 4) {
    asm("ld.global.nc.v4.u32 {%0, %1, %2, %3}, [%4];"
        : "=r"(b.w[0]), "=r"(b.w[1]), "=r"(b.w[2]), "=r"(b.w[3])
        : "l"(p));
  } else {
#pragma unroll
    for (uint32_t i = 0; i < kNearWords; i += 8)
      asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
          : "=r"(b.w[i]), "=r"(b.w[i + 1]), "=r"(b.w[i + 2]), "=r"(b.w[i + 3]),
            "=r"(b.w[i + 4]), "=r"(b.w[i + 5]), "=r"(b.w[i + 6]), "=r"(b.w[i + 7])
          : "l"(p + i));
  }
  return b;
}
__device__ __forceinline__ bool bucket16_has(const NearBucket &b, uint32_t kk) {
  uint32_t z = 0;
#pragma unroll
  for (uint32_t i = 0; i < kNearWords; ++i) {
    const uint32_t y = b.w[i] ^ kk;
    z |= (y - 0x10001u) & ~y;
  }
  return (z & 0x80008000u) != 0;
}
__device__ __forceinline__ bool bucket16_full(const NearBucket &b) {
  return (b.w[kNearWords - 1] >> 16) != kNearEmpty;
}
// The buckets after bucket bk of a near row, for a lookup whose first
// bucket was full and did not hold the key.
__device__ __forceinline__ bool near_contains_rest(const uint32_t *rowtab,
                                                uint32_t nbk, uint32_t bk,
                                                uint32_t kk) {
  for (uint32_t probe = 1; probe < nbk; ++probe) {
    bk = bk + 1 == nbk ? 0 : bk + 1;
    const NearBucket b = ld_bucket16(rowtab + (uint64_t)bk * kNearWords);
    if (bucket16_has(b, kk)) return true;
    if (!bucket16_full(b)) return false;
  }
  return false;
}

// Per-row {first bucket, buckets} from the bucket prefix (total < 2^32), so
// a lookup reads its row's set with one 8-byte load.
__global__ void k_hash_rows(const uint64_t *__restrict__ hoff, uint64_t n,
                            uint2 *__restrict__ rows) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x)
    rows[v] = make_uint2((uint32_t)hoff[v], (uint32_t)(hoff[v + 1] - hoff[v]));
}

__device__ __forceinline__ uint32_t hash_bucket(uint32_t x, uint32_t nbk) {
  return __umulhi(x * kHashMul, nbk);
}

// Buckets of a row with out-degree d (0 below min_degree); keys_per_bucket
// <= kHashBucket, so a row's buckets always have room for all its columns.
__host__ __device__ __forceinline__ uint32_t hash_buckets_for(
    uint64_t d, uint32_t min_degree, uint32_t keys_per_bucket) {
  if (d < min_degree || d == 0) return 0;
  return (uint32_t)((d + keys_per_bucket - 1) / keys_per_bucket);
}

// The 8 slots of one bucket in one 32-byte load (p 32-byte aligned).
struct Bucket {
  uint32_t s0, s1, s2, s3, s4, s5, s6, s7;
};
__device__ __forceinline__ Bucket ld_bucket(const uint32_t *p) {
  Bucket b;
  asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=r"(b.s0), "=r"(b.s1), "=r"(b.s2), "=r"(b.s3), "=r"(b.s4),
        "=r"(b.s5), "=r"(b.s6), "=r"(b.s7)
      : "l"(p));
  return b;
}
__device__ __forceinline__ bool bucket_has(const Bucket &b, uint32_t u) {
  return b.s0 == u || b.s1 == u || b.s2 == u || b.s3 == u || b.s4 == u ||
         b.s5 == u || b.s6 == u || b.s7 == u;
}

template <typename Off>
__global__ void k_hash_sizes(const Off *__restrict__ rp, uint64_t n,
                             uint64_t first_excluded, uint32_t min_degree,
                             uint32_t keys_per_bucket,
                             uint32_t *__restrict__ nb) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x)
    nb[v] = v < first_excluded
                ? hash_buckets_for(ld_off(rp, v + 1) - ld_off(rp, v),
                                   min_degree, keys_per_bucket)
                : 0u;
}

// Slots in use of a bucket under construction (they fill in order, so the
// count of non-empty slots is the fill): two 16-byte volatile loads, both
// in flight, instead of a chain of up to eight slot reads. The bucket's
// slots were written by this warp before its last __syncwarp.
__device__ __forceinline__ uint32_t bucket_fill(const uint32_t *q) {
  uint32_t a0, a1, a2, a3, b0, b1, b2, b3;
  asm volatile("ld.volatile.global.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(a0), "=r"(a1), "=r"(a2), "=r"(a3) : "l"(q));
  asm volatile("ld.volatile.global.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(b0), "=r"(b1), "=r"(b2), "=r"(b3) : "l"(q + 4));
  return (a0 != kHashEmpty) + (a1 != kHashEmpty) + (a2 != kHashEmpty) +
         (a3 != kHashEmpty) + (b0 != kHashEmpty) + (b1 != kHashEmpty) +
         (b2 != kHashEmpty) + (b3 != kHashEmpty);
}

// One warp per row, no atomics: the row's columns go in rounds of 32;
// lanes whose columns share a bucket (__match_any_sync) take consecutive
// slots after the bucket's current fill, read once by the group's first
// lane. Lanes that find the bucket full continue one at a time into the
// following buckets. The warp is the row's only writer, so plain stores
// ordered by __syncwarp suffice. Columns of a row are distinct and the
// buckets have room for all of them.
// Rows [v_begin, min(v_end, n)).
template <typename Off>
__global__ void k_hash_build(const Off *__restrict__ rp,
                             const uint32_t *__restrict__ ci, uint64_t n,
                             const uint64_t *__restrict__ hoff,
                             uint32_t *__restrict__ tab, uint64_t v_begin = 0,
                             uint64_t v_end = ~0ull) {
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t end = v_end < n ? v_end : n;
  for (uint64_t v = v_begin + warp; v < end; v += nwarps) {
    const uint64_t b0 = hoff[v];
    const uint32_t nbk = (uint32_t)(hoff[v + 1] - b0);
    if (nbk == 0) continue;
    uint32_t *rowtab = tab + b0 * kHashBucket;
    const uint64_t e = ld_off(rp, v + 1);
    for (uint64_t j0 = ld_off(rp, v); j0 < e; j0 += 32) {
      const uint64_t j = j0 + lane;
      const bool valid = j < e;
      const uint32_t x = valid ? ci[j] : 0u;
      const uint32_t bk = valid ? hash_bucket(x, nbk) : 0xFFFFFFFFu;
      const uint32_t peers = __match_any_sync(0xffffffffu, bk);
      const uint32_t leader = __ffs(peers) - 1;
      const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
      uint32_t fill = 0;
      if (valid && lane == leader) fill = bucket_fill(rowtab + (uint64_t)bk * kHashBucket);
      fill = __shfl_sync(0xffffffffu, fill, leader);
      const uint32_t slot = fill + rank;
      if (valid && slot < kHashBucket) rowtab[(uint64_t)bk * kHashBucket + slot] = x;
      __syncwarp();
      uint32_t over = __ballot_sync(0xffffffffu, valid && slot >= kHashBucket);
      while (over) {
        const uint32_t l = __ffs(over) - 1;
        if (lane == l) {
          uint32_t b = bk;
          for (uint32_t probe = 1; probe < nbk; ++probe) {
            b = b + 1 == nbk ? 0 : b + 1;
            uint32_t *q = rowtab + (uint64_t)b * kHashBucket;
            const uint32_t f = bucket_fill(q);
            if (f < kHashBucket) {
              q[f] = x;
              break;
            }
          }
        }
        __syncwarp();
        over &= over - 1;
      }
    }
  }
}

// Slots in use of a near bucket under construction: one volatile load per
// 16 bytes, counting the 16-bit slots that are not 0xFFFF.
__device__ __forceinline__ uint32_t bucket16_fill(const uint16_t *q) {
  uint32_t f = 0;
#pragma unroll
  for (uint32_t i = 0; i < kNearWords; i += 4) {
    uint32_t w0, w1, w2, w3;
    asm volatile("ld.volatile.global.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(w0), "=r"(w1), "=r"(w2), "=r"(w3)
                 : "l"(reinterpret_cast<const uint32_t *>(q) + i));
    for (uint32_t x : {w0, w1, w2, w3})
      f += ((x & 0xFFFFu) != kNearEmpty) + ((x >> 16) != kNearEmpty);
  }
  return f;
}

// k_hash_build for the near rows v = first + r, r_begin <= r < count: the
// same atomic-free warp build with 16-bit keys v's columns x store as
// x - v - 1 (columns outside (v, n) are never looked up and are left out).
template <typename Off>
__global__ void k_near_build(const Off *__restrict__ rp,
                             const uint32_t *__restrict__ ci, uint64_t n,
                             uint64_t first, uint64_t count,
                             const uint64_t *__restrict__ noff,
                             uint32_t *__restrict__ ntab,
                             uint64_t r_begin = 0) {
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t r = r_begin + warp; r < count; r += nwarps) {
    const uint64_t v = first + r;
    const uint64_t b0 = noff[r];
    const uint32_t nbk = (uint32_t)(noff[r + 1] - b0);
    if (nbk == 0) continue;
    uint16_t *rowtab = reinterpret_cast<uint16_t *>(ntab + b0 * kNearWords);
    const uint64_t e = ld_off(rp, v + 1);
    for (uint64_t j0 = ld_off(rp, v); j0 < e; j0 += 32) {
      const uint64_t j = j0 + lane;
      const uint32_t x = j < e ? ci[j] : 0u;
      const bool valid = j < e && x > v && x < n;
      const uint32_t key = valid ? (uint32_t)(x - v - 1) : 0u;
      const uint32_t bk = valid ? hash_bucket(key, nbk) : 0xFFFFFFFFu;
      const uint32_t peers = __match_any_sync(0xffffffffu, bk);
      const uint32_t leader = __ffs(peers) - 1;
      const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
      uint32_t fill = 0;
      if (valid && lane == leader) fill = bucket16_fill(rowtab + (uint64_t)bk * kNearSlots);
      fill = __shfl_sync(0xffffffffu, fill, leader);
      const uint32_t slot = fill + rank;
      if (valid && slot < kNearSlots)
        rowtab[(uint64_t)bk * kNearSlots + slot] = (uint16_t)key;
      __syncwarp();
      uint32_t over = __ballot_sync(0xffffffffu, valid && slot >= kNearSlots);
      while (over) {
        const uint32_t l = __ffs(over) - 1;
        if (lane == l) {
          uint32_t b = bk;
          for (uint32_t probe = 1; probe < nbk; ++probe) {
            b = b + 1 == nbk ? 0 : b + 1;
            uint16_t *q = rowtab + (uint64_t)b * kNearSlots;
            const uint32_t f = bucket16_fill(q);
            if (f < kNearSlots) {
              q[f] = (uint16_t)key;
              break;
            }
          }
        }
        __syncwarp();
        over &= over - 1;
      }
    }
  }
}

// The buckets after bucket bk of a row (nbk buckets at rowtab), for a
// lookup whose first bucket was full and did not hold u.
__device__ __forceinline__ bool hash_contains_rest(const uint32_t *rowtab,
                                                uint32_t nbk, uint32_t bk,
                                                uint32_t u) {
  for (uint32_t probe = 1; probe < nbk; ++probe) {
    bk = bk + 1 == nbk ? 0 : bk + 1;
    const Bucket b = ld_bucket(rowtab + (uint64_t)bk * kHashBucket);
    if (bucket_has(b, u)) return true;
    if (b.s7 == kHashEmpty) return false;  // slots fill in order
  }
  return false;
}

// Is u in the set of row w (nbk buckets from b0)? Bounded by nbk buckets.
__device__ __forceinline__ bool hash_contains(const uint32_t *__restrict__ tab,
                                              uint64_t b0, uint32_t nbk,
                                              uint32_t u) {
  const uint32_t *rowtab = tab + b0 * kHashBucket;
  const uint32_t bk = hash_bucket(u, nbk);
  const Bucket b = ld_bucket(rowtab + (uint64_t)bk * kHashBucket);
  if (bucket_has(b, u)) return true;
  if (b.s7 == kHashEmpty) return false;
  return hash_contains_rest(rowtab, nbk, bk, u);
}

// Is key t (= u - w - 1 <= 65534) in the near set of row w (nbk 16-byte
// buckets from b0)? Bounded by nbk buckets.
__device__ __forceinline__ bool near_contains(const uint32_t *__restrict__ ntab,
                                              uint64_t b0, uint32_t nbk,
                                              uint32_t t) {
  const uint32_t *rowtab = ntab + b0 * kNearWords;
  const uint32_t kk = t * 0x10001u;
  const uint32_t bk = hash_bucket(t, nbk);
  const NearBucket b = ld_bucket16(rowtab + (uint64_t)bk * kNearWords);
  if (bucket16_has(b, kk)) return true;
  if (!bucket16_full(b)) return false;
  return near_contains_rest(rowtab, nbk, bk, kk);
}

// Layout of the dense core bit matrix (see k_core_count below), also used
// as the count's bitmap when the core covers the bitmap's rows.
constexpr uint32_t kCoreMaxH4 = 2048;  // h <= 65536: 8 KB bit row per block
constexpr uint32_t kCoreBlock = 256;

__host__ __device__ __forceinline__ uint32_t core_row_first(uint32_t r) {
  return (r >> 7) << 2;
}
// First word of row r: rows of group q = r >> 5 hold H4 - 4 (q >> 2) words.
__host__ __device__ __forceinline__ uint64_t core_row_off(uint32_t H4,
                                                         uint32_t r) {
  const uint64_t q = r >> 5, Q = q >> 2, R = q & 3;
  const uint64_t S = 2 * Q * (Q ? Q - 1 : 0) + R * Q;  // sum of (q' >> 2), q' < q
  return 32 * (q * H4 - 4 * S) + (uint64_t)(r & 31) * (H4 - 4 * Q);
}

// Edge check of one wedge (v; w, u): the bitmap bit when w is in the
// bitmap range, else u searched in N+(w) -- in the warp's shared-memory
// stage when it holds N+(w) (kStage), in global memory otherwise. The
// warp stages N+(w) of its last searching lane when it differs from the
// staged row and fits kStageCap. All lanes must call this together.
template <typename Off, bool kBatch, bool kStage, bool kHash = false,
          bool kNear = false, bool kAligned = false>
__device__ __forceinline__ uint32_t check_wedge(
    const Off *__restrict__ rp, const uint32_t *__restrict__ ci, uint64_t n,
    const uint32_t *__restrict__ bm, uint64_t bm_first, uint64_t S,
    const BatchView &bv, bool ok, uint32_t g, uint32_t w, uint32_t u,
    uint32_t *buf, uint64_t &staged, uint32_t &staged_d,
    const HashView &hv = HashView{}) {
  const int lane = threadIdx.x & 31;
  bool is_bm;
  uint32_t hit = 0;
  if (kBatch) {
    // Union ids, n_g and local ids are below 2^32 (batch_create checks the
    // union's size), so the graph's frame is 32-bit.
    uint32_t vb = 0, ng = 0, bmf = 0;
    uint64_t Sg = 0, bmo = 0;
    if (ok) {
      const Bucket gi = ld_bucket(bv.ginfo + (uint64_t)g * 8);
      vb = gi.s0;
      ng = gi.s1;
      bmf = gi.s2;
      bmo = gi.s3 | ((uint64_t)gi.s4 << 32);
      Sg = gi.s5 | ((uint64_t)gi.s6 << 32);
    }
    const uint32_t wl = w - vb, ul = u - vb;
    is_bm = ok && w >= vb && wl < ng && wl >= bmf;
    if (is_bm && u > w && ul < ng) {
      const uint32_t nw = ng - wl;
      const uint64_t idx = Sg - (((uint64_t)nw * (nw - 1)) >> 1) + (ul - wl - 1);
      if (idx < Sg)
        hit = (ld_bitmap(bm + bmo + (idx >> 5), l2_evict_last_policy()) >>
               ((uint32_t)idx & 31)) & 1u;
    }
  } else {
    // n < 2^32, so ids and n - w fit 32 bits; (n - w)(n - w - 1) is one
    // 32 x 32 -> 64-bit multiply.
    const uint32_t n32 = (uint32_t)n;
    is_bm = ok && (uint64_t)w >= bm_first;
    if (is_bm && u > w && u < n32) {
      if (kAligned) {
        // the core matrix: row w - bm_first, column u - bm_first (S = H4)
        const uint32_t r = w - (uint32_t)bm_first, c = u - (uint32_t)bm_first;
        const uint64_t word = core_row_off((uint32_t)S, r) - core_row_first(r) + (c >> 5);
        hit = (ld_bitmap(bm + word, l2_evict_last_policy()) >> (c & 31)) & 1u;
      } else {
        const uint32_t nw = n32 - w;
        const uint64_t idx = S - (((uint64_t)nw * (nw - 1)) >> 1) + (u - w - 1);
        if (idx < S)
          hit = (ld_bitmap(bm + (idx >> 5), l2_evict_last_policy()) >> ((uint32_t)idx & 31)) & 1u;
      }
    }
  }
  const bool is_srch = ok && !is_bm && (uint64_t)w < n;
  if (kStage) {
    const uint32_t smask = __ballot_sync(0xffffffffu, is_srch);
    if (smask) {
      const int src = 31 - __clz(smask);
      const uint32_t wc = __shfl_sync(0xffffffffu, w, src);
      if ((uint64_t)wc != staged) {
        const uint64_t bw = ld_off(rp, wc);
        const uint64_t dw = ld_off(rp, wc + 1) - bw;
        if (dw <= (uint64_t)kStageCap) {
          __syncwarp();
          for (uint32_t q = lane; q < dw; q += 32) buf[q] = __ldg(ci + bw + q);
          __syncwarp();
          staged = wc;
          staged_d = (uint32_t)dw;
        }
      }
    }
  }
  if (kNear && is_srch && w - hv.nfirst < hv.ncount) {
    const uint2 hr = __ldg(hv.nrows + (w - hv.nfirst));
    if (hr.y) {
      const uint32_t t = u - w - 1;  // wraps for u <= w
      if (t >= (uint32_t)n - w - 1) return 0u;
      return near_contains(hv.ntab, hr.x, hr.y, t) ? 1u : 0u;
    }
  } else if (kHash && is_srch && hv.rows) {
    const uint2 hr = __ldg(hv.rows + w);
    if (hr.y) return hash_contains(hv.tab, hr.x, hr.y, u) ? 1u : 0u;
  }
  if (is_srch) {
    if (kStage && (uint64_t)w == staged) {
      uint32_t len = staged_d;
      if (len > 0) {
        uint32_t p = 0;
        while (len > 1) {
          const uint32_t h = len >> 1;
          p = (buf[p + h] <= u) ? p + h : p;
          len -= h;
        }
        hit = buf[p] == u ? 1u : 0u;
      }
    } else {
      // Out-degrees are below 2^30: the search runs on a 32-bit offset
      // from the row start.
      const uint32_t *row = ci + ld_off(rp, w);
      uint32_t len = (uint32_t)(ld_off(rp, w + 1) - ld_off(rp, w));
      if (len > 0) {
        uint32_t lo = 0;
        while (len > 1) {
          const uint32_t h = len >> 1;
          lo = (__ldg(row + lo + h) <= u) ? lo + h : lo;
          len -= h;
        }
        hit = (__ldg(row + lo) == u) ? 1u : 0u;
      }
    }
  }
  return hit;
}

// Hits of one row segment: the nseg wedges (v; w, up[k]), k < nseg, of a
// single row of N+(v) -- w is the same for the whole warp, so the choice of
// check and its per-row constants are computed once, and each lane only
// loads its u (coalesced) and probes; lanes past nseg in the last round
// stay idle. Columns outside the graph (or u <= w, which a sorted oriented
// row never has) count nothing.
constexpr uint32_t kSegMinRow = 16;
template <typename Off, bool kBatch, bool kHash, bool kNear = false,
          bool kAligned = false>
__device__ __forceinline__ uint32_t segment_hits(
    const Off *__restrict__ rp, const uint32_t *__restrict__ ci, uint64_t n,
    const uint32_t *__restrict__ bm, uint64_t bm_first, uint64_t S,
    const BatchView &bv, uint32_t g, const HashView &hv, uint32_t w,
    const uint32_t *__restrict__ up, uint32_t nseg) {
  const uint32_t lane = threadIdx.x & 31;
  uint64_t vb = 0, ng = n, bmf = bm_first, Sg = S;
  const uint32_t *bmg = bm;
  if (kBatch) {
    const Bucket gi = ld_bucket(bv.ginfo + (uint64_t)g * 8);
    vb = gi.s0;
    ng = gi.s1;
    bmf = gi.s2;
    bmg = bm + (gi.s3 | ((uint64_t)gi.s4 << 32));
    Sg = gi.s5 | ((uint64_t)gi.s6 << 32);
  }
  const uint64_t wl = (uint64_t)w - vb;
  if (w < vb || wl >= ng) return 0;
  uint32_t hits = 0;
  if (wl >= bmf) {
    // Bitmap row of w: bit rowbit + (u - w - 1) for w < u < vb + ng; the
    // row ends where row w + 1 starts, nw - 1 bits later. With the core
    // matrix as the bitmap (kAligned, Sg = H4): row r = w - bmf indexes
    // column c = u - bmf = (u - w - 1) + r + 1 from its column-0 word.
    const uint64_t nw = ng - wl;
    const uint32_t *words;
    uint32_t sh;
    if (kAligned && !kBatch) {
      const uint32_t r = (uint32_t)(wl - bmf);
      words = bmg + core_row_off((uint32_t)Sg, r) - core_row_first(r);
      sh = r + 1;
    } else {
      const uint64_t rowbit = Sg - nw * (nw - 1) / 2;
      words = bmg + (rowbit >> 5);
      sh = (uint32_t)rowbit & 31u;
    }
    const uint32_t lim = (uint32_t)(nw - 1);
    const uint64_t pol = l2_evict_last_policy();
#pragma unroll 4
    for (uint32_t k = lane; k < nseg; k += 32) {
      const uint32_t u = __ldg(up + k);
      const uint32_t t = u - w - 1;
      if (t < lim) {
        const uint32_t x = t + sh;
        hits += (ld_bitmap(words + (x >> 5), pol) >> (x & 31u)) & 1u;
      }
    }
    return hits;
  }
  if (kNear && w - hv.nfirst < hv.ncount) {
    // Near set of w: keys t = u - w - 1; a column outside (w, n) (t >= lim)
    // still reads an in-range bucket but counts nothing.
    const uint2 hr = __ldg(hv.nrows + (w - hv.nfirst));
    const uint32_t nbk = hr.y;
    if (nbk) {
      const uint32_t *rowtab = hv.ntab + (uint64_t)hr.x * kNearWords;
      const uint32_t lim = (uint32_t)n - w - 1;
      uint32_t k = lane;
      // three rounds at a time: three buckets in flight before any compare
      // (16-byte buckets leave room for a third without spilling)
      for (; k + 64 < nseg; k += 96) {
        uint32_t t[3], bq[3];
        NearBucket b[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          t[q] = __ldg(up + k + 32 * q) - w - 1;
          bq[q] = hash_bucket(t[q], nbk);
        }
#pragma unroll
        for (int q = 0; q < 3; ++q) b[q] = ld_bucket16(rowtab + (uint64_t)bq[q] * kNearWords);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const uint32_t kk = t[q] * 0x10001u;
          const bool in = t[q] < lim;
          bool h = in && bucket16_has(b[q], kk);
          if (in && !h && bucket16_full(b[q])) h = near_contains_rest(rowtab, nbk, bq[q], kk);
          hits += h ? 1u : 0u;
        }
      }
      for (; k < nseg; k += 32) {
        const uint32_t t = __ldg(up + k) - w - 1;
        const uint32_t bk = hash_bucket(t, nbk);
        const NearBucket b = ld_bucket16(rowtab + (uint64_t)bk * kNearWords);
        const uint32_t kk = t * 0x10001u;
        const bool in = t < lim;
        bool h = in && bucket16_has(b, kk);
        if (in && !h && bucket16_full(b)) h = near_contains_rest(rowtab, nbk, bk, kk);
        hits += h ? 1u : 0u;
      }
      return hits;
    }
  } else if (kHash && hv.rows) {
    const uint2 hr = __ldg(hv.rows + w);
    const uint64_t b0 = hr.x;
    const uint32_t nbk = hr.y;
    if (nbk) {
      const uint32_t *rowtab = hv.tab + b0 * kHashBucket;
      uint32_t k = lane;
      // two rounds at a time: both buckets in flight before either compare
      for (; k + 32 < nseg; k += 64) {
        const uint32_t u0 = __ldg(up + k), u1 = __ldg(up + k + 32);
        const uint32_t k0 = hash_bucket(u0, nbk), k1 = hash_bucket(u1, nbk);
        const Bucket b0 = ld_bucket(rowtab + (uint64_t)k0 * kHashBucket);
        const Bucket b1 = ld_bucket(rowtab + (uint64_t)k1 * kHashBucket);
        bool h0 = bucket_has(b0, u0), h1 = bucket_has(b1, u1);
        const bool more0 = !h0 && b0.s7 != kHashEmpty;
        const bool more1 = !h1 && b1.s7 != kHashEmpty;
        if (more0) h0 = hash_contains_rest(rowtab, nbk, k0, u0);
        if (more1) h1 = hash_contains_rest(rowtab, nbk, k1, u1);
        hits += (h0 ? 1u : 0u) + (h1 ? 1u : 0u);
      }
      if (k < nseg) {
        const uint32_t u = __ldg(up + k);
        const uint32_t bk = hash_bucket(u, nbk);
        const Bucket b = ld_bucket(rowtab + (uint64_t)bk * kHashBucket);
        bool h = bucket_has(b, u);
        if (!h && b.s7 != kHashEmpty) h = hash_contains_rest(rowtab, nbk, bk, u);
        hits += h ? 1u : 0u;
      }
      return hits;
    }
  }
  // Binary search in N+(w); the row length is warp-uniform, so is the loop.
  const uint64_t rbw = ld_off(rp, w);
  const uint32_t len0 = (uint32_t)(ld_off(rp, w + 1) - rbw);
  if (len0 == 0) return 0;
  const uint32_t *row = ci + rbw;
  for (uint32_t k = lane; k < nseg; k += 32) {
    const uint32_t u = __ldg(up + k);
    uint32_t lo = 0, len = len0;
    while (len > 1) {
      const uint32_t h = len >> 1;
      lo = (__ldg(row + lo + h) <= u) ? lo + h : lo;
      len -= h;
    }
    hits += (__ldg(row + lo) == u) ? 1u : 0u;
  }
  return hits;
}

// One warp's tile t of the row-walk count (the body of k_count_rows; the
// resident serving kernel calls it with each graph's parameters): the warp
// walks the tile's wedges and adds its hits to acc (a batch flushes them per
// graph into bv.counts as it goes).
template <typename Off, bool kBatch, bool kStage, bool kHash, bool kSegs, bool kNear,
          bool kAligned = false>
__device__ __forceinline__ void rows_tile(
    const Off *__restrict__ rp, const uint32_t *__restrict__ ci, uint64_t n,
    const uint64_t *__restrict__ act_wp, const uint64_t *__restrict__ act_rb,
    const uint32_t *__restrict__ act_d, uint64_t K,
    const uint32_t *__restrict__ tile_k, uint64_t t, uint64_t wb, uint64_t we,
    uint64_t G, const uint32_t *__restrict__ bm, uint64_t bm_first, uint64_t S,
    const BatchView &bv, const HashView &hv, uint32_t *buf, uint64_t &staged,
    uint32_t &staged_d, uint64_t &acc, uint32_t &cur_g) {
  const int lane = threadIdx.x & 31;
  uint64_t base, end;
  tile_bounds<kBatch>(t, wb, we, G, bv, &base, &end);
  // Warp-uniform position of wedge `base`.
  uint64_t kcur = tile_k[t];
  uint64_t rb = __ldg(act_rb + kcur);
  uint32_t d = __ldg(act_d + kcur);
  uint32_t wi = 0, ui = 1;
  bool pos_ok = decode_wedge(base - __ldg(act_wp + kcur), d, &wi, &ui);
  uint32_t gv = kBatch ? __ldg(bv.act_g + kcur) : 0u;
  uint32_t c = 0;
  while (base < end && pos_ok) {
    if (kSegs && d - ui >= kSegMinRow) {
      // Long-row segment: the rest of row wi (or of the tile), in rounds
      // of 32 wedges; the last round may leave lanes idle, which costs
      // less than a per-lane round when the row has kSegMinRow or more
      // wedges left.
      const uint64_t left = end - base;
      const uint32_t rem = d - ui;
      const uint32_t nseg = (uint32_t)(left < rem ? left : rem);
      const uint32_t w = __ldg(ci + rb + wi);
      if (kBatch && gv != cur_g) {
        flush_count(c, cur_g != 0xFFFFFFFFu ? bv.counts + cur_g : nullptr);
        acc += c;
        c = 0;
        cur_g = gv;
      }
      c += segment_hits<Off, kBatch, kHash, kNear, kAligned>(
          rp, ci, n, bm, bm_first, S, bv, gv, hv, w, ci + rb + ui, nseg);
      base += nseg;
      ui += nseg;
      if (ui == d) {
        // Row wi ended; rem >= kSegMinRow leaves row wi + 1 non-empty.
        wi += 1;
        ui = wi + 1;
      }
      continue;
    }
    const uint32_t n_round = (uint32_t)(end - base < 32 ? end - base : 32);
    const uint32_t rem0 = d - ui;                      // left in row wi
    const uint32_t len1 = wi + 2 < d ? d - wi - 2 : 0;  // row wi + 1
    const bool valid = lane < (int)n_round;
    bool ok = valid;
    uint32_t w = 0, u = 0, g = gv;
    if (n_round <= rem0 + len1) {
      // Fast round: rows wi and wi + 1 of vertex kcur.
      const bool in1 = (uint32_t)lane >= rem0;
      const uint32_t my_ui = in1 ? wi + 2 + ((uint32_t)lane - rem0) : ui + lane;
      const uint32_t w0 = __ldg(ci + rb + wi);
      const uint32_t w1 = n_round > rem0 ? __ldg(ci + rb + wi + 1) : 0u;
      w = in1 ? w1 : w0;
      if (valid) u = __ldg(ci + rb + my_ui);
      if (n_round < rem0) {
        ui += n_round;
      } else {
        const uint32_t c1 = n_round - rem0;
        if (c1 < len1) {
          wi += 1;
          ui = wi + 1 + c1;
        } else if (wi + 3 < d) {
          wi += 2;
          ui = wi + 1;
        } else if (base + n_round < end) {
          kcur += 1;
          rb = __ldg(act_rb + kcur);
          d = __ldg(act_d + kcur);
          wi = 0;
          ui = 1;
          if (kBatch) gv = __ldg(bv.act_g + kcur);
        }
      }
    } else {
      // General round: vertex window + per-lane decode.
      const uint64_t i = base + lane;
      const uint64_t kl = kcur + lane;
      const uint64_t E = kl <= K ? __ldg(act_wp + kl) : ~0ull;
      const uint64_t RB = kl < K ? __ldg(act_rb + kl) : 0;
      const uint32_t D = kl < K ? __ldg(act_d + kl) : 2u;
      uint32_t GW = 0;
      if (kBatch) GW = kl < K ? __ldg(bv.act_g + kl) : 0u;
      // The search runs on prefix entries relative to base, saturated to
      // 32 bits: only "entry <= base + lane" (lane < 32) matters.
      const uint32_t Er = E <= base ? 0u
                          : (E - base > 0xFFFFFFFFull ? 0xFFFFFFFFu
                                                      : (uint32_t)(E - base));
      uint32_t j = 0;
#pragma unroll
      for (uint32_t step = 16; step > 0; step >>= 1) {
        const uint32_t e = __shfl_sync(0xffffffffu, Er, j + step);
        if (e <= (uint32_t)lane) j += step;
      }
      const uint64_t e0 = __shfl_sync(0xffffffffu, E, j);
      const uint64_t rbl = __shfl_sync(0xffffffffu, RB, j);
      const uint64_t dl = __shfl_sync(0xffffffffu, D, j);
      if (kBatch) g = __shfl_sync(0xffffffffu, GW, j);
      const uint32_t j31 = __shfl_sync(0xffffffffu, j, 31);
      uint32_t wl = 0, ul = 0;
      if (valid) {
        ok = e0 <= i && decode_wedge(i - e0, dl, &wl, &ul);
        if (ok) {
          w = __ldg(ci + rbl + wl);
          u = __ldg(ci + rbl + ul);
        }
      }
      if (base + n_round < end) {
        // n_round == 32 here: the next round starts at the successor of
        // lane 31's wedge (vertex kcur + j31, row wl, column ul) in wedge
        // order -- the next column, the next row, or the first wedge of
        // the next active vertex, whose row start and degree the window
        // already holds unless it is entry 32.
        const uint32_t w31 = __shfl_sync(0xffffffffu, wl, 31);
        const uint32_t u31 = __shfl_sync(0xffffffffu, ul, 31);
        const uint32_t d31 = __shfl_sync(0xffffffffu, (uint32_t)dl, 31);
        pos_ok = __shfl_sync(0xffffffffu, ok ? 1u : 0u, 31) != 0;
        uint32_t adv = j31;
        if (u31 + 1 < d31) {
          wi = w31;
          ui = u31 + 1;
        } else if (w31 + 2 < d31) {
          wi = w31 + 1;
          ui = w31 + 2;
        } else {
          wi = 0;
          ui = 1;
          adv = j31 + 1;
        }
        if (adv < 32) {
          rb = __shfl_sync(0xffffffffu, RB, adv);
          d = __shfl_sync(0xffffffffu, D, adv);
          if (kBatch) gv = __shfl_sync(0xffffffffu, GW, adv);
        } else {
          rb = __ldg(act_rb + kcur + 32);
          d = __ldg(act_d + kcur + 32);
          if (kBatch) gv = __ldg(bv.act_g + kcur + 32);
        }
        kcur += adv;
      }
    }
    uint32_t hit = check_wedge<Off, kBatch, kStage, kHash, kNear, kAligned>(
        rp, ci, n, bm, bm_first, S, bv, ok, g, w, u, buf, staged, staged_d, hv);
    if (kBatch) {
      const uint32_t g0 = __shfl_sync(0xffffffffu, g, 0);
      const bool uni = __all_sync(0xffffffffu, !ok || g == g0);
      if (!(uni && g0 == cur_g)) {
        flush_count(c, cur_g != 0xFFFFFFFFu ? bv.counts + cur_g : nullptr);
        acc += c;
        c = 0;
        cur_g = 0xFFFFFFFFu;
        if (uni) {
          cur_g = g0;
        } else {
          const uint32_t key = ok ? g : 0xFFFFFFFFu;
          const uint32_t peers = __match_any_sync(0xffffffffu, key);
          const uint32_t hits = __ballot_sync(0xffffffffu, hit) & peers;
          if (ok && lane == __ffs(peers) - 1 && hits)
            atomicAdd(bv.counts + g, (unsigned long long)__popc(hits));
          acc += hit;
          hit = 0;
        }
      }
    }
    c += hit;
    base += n_round;
  }
  if (kBatch) {
    flush_count(c, cur_g != 0xFFFFFFFFu ? bv.counts + cur_g : nullptr);
    cur_g = 0xFFFFFFFFu;
  }
  acc += c;
}

// Row-walk count. Each warp takes whole tiles of G = 256 * s consecutive
// wedges from a global counter. Inside a tile it keeps the position of its
// next wedge -- active vertex k, row w_i, column u_i -- in warp-uniform
// registers (one decode per tile) and walks it in rounds of 32 lanes:
//   * fast round: the 32 wedges lie in rows w_i and w_i + 1 of the same
//     vertex (the common case on skewed graphs: rows are long); lane l
//     takes column u_i + l, or the matching column of row w_i + 1, so a
//     lane needs two adds and one coalesced load of u;
//   * general round (short rows, vertex ends): the 32-entry vertex window
//     and the per-lane decode of the warp-staged kernel, then the position
//     of the next wedge is decoded once, warp-uniformly.
// The check and the per-graph accumulation are those of k_count_staged.
template <typename Off, bool kBatch, bool kStage, int kMinBlocks = 1,
          bool kHash = false, bool kSegs = false, bool kNear = false,
          bool kAligned = false>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, kMinBlocks)
    k_count_rows(const Off *__restrict__ rp, const uint32_t *__restrict__ ci,
                 uint64_t n, const uint64_t *__restrict__ act_wp,
                 const uint64_t *__restrict__ act_rb,
                 const uint32_t *__restrict__ act_d, uint64_t K,
                 const uint32_t *__restrict__ tile_k, uint64_t tiles,
                 uint64_t wb, uint64_t we, uint64_t G,
                 const uint32_t *__restrict__ bm, uint64_t bm_first,
                 uint64_t S, unsigned long long *__restrict__ next_tile,
                 unsigned long long *__restrict__ out, BatchView bv,
                 HashView hv = HashView{}) {
  __shared__ uint32_t stage[kStage ? kWarpsPerBlock : 1][kStage ? kStageCap : 1];
  __shared__ unsigned long long warp_acc[kWarpsPerBlock];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t *buf = stage[kStage ? warp : 0];
  uint64_t staged = ~0ull;
  uint32_t staged_d = 0;
  uint64_t acc = 0;
  uint32_t cur_g = 0xFFFFFFFFu;
  // With a tile counter the grid is persistent: warps take tiles until none
  // are left. Without one (next_tile == nullptr) every warp counts the one
  // tile blockIdx.x * kWarpsPerBlock + warp and its block ends, so blocks of
  // other streams get the SMs as this launch drains.
  bool taken = false;
  for (;;) {
    unsigned long long t = 0;
    if (next_tile) {
      if (lane == 0) t = atomicAdd(next_tile, 1ull);
      t = __shfl_sync(0xffffffffu, t, 0);
    } else {
      if (taken) break;
      taken = true;
      t = (unsigned long long)blockIdx.x * kWarpsPerBlock + warp;
    }
    if (t >= tiles) break;
    rows_tile<Off, kBatch, kStage, kHash, kSegs, kNear, kAligned>(
        rp, ci, n, act_wp, act_rb, act_d, K, tile_k, t, wb, we, G, bm, bm_first, S,
        bv, hv, buf, staged, staged_d, acc, cur_g);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) warp_acc[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long tot = 0;
    for (int q = 0; q < kWarpsPerBlock; ++q) tot += warp_acc[q];
    if (tot) atomicAdd(out, tot);
  }
}

// ---------------------------------------------------------------------------
// Dense core. With the degree order, the top h vertices [v0, v0 + h) are
// the graph's hubs, and every out-neighbour of a core vertex is a core
// vertex (columns of row v are > v). So the triangles closed by all wedges
// of a core vertex v are sum over w in N+(v) of |N+(v) & N+(w)|, and with
// the core rows as bit rows that is a popcount of row AND row -- 32 columns
// per word instead of one edge check per wedge. The wedges (v; w, u) with
// u in N+(v), u > w of one pair (v, w) are exactly N+(v) & N+(w) (the row
// of w holds only columns > w), so the pair's wedge range maps to whole
// words; a wedge range that cuts a pair (at most its first and last pair)
// masks the columns of the pair's cut.
//
// Layout: local ids r = v - v0 in [0, h); H4 = ceil(h / 32) rounded up to a
// multiple of 4 words. Row r holds word columns [4 (r >> 7), H4): word jj
// has the columns [32 jj, 32 jj + 32), so every row is 16-byte aligned, all
// rows index columns the same way (a row AND needs no shifts), and the
// words below the row's first column stay zero.
// One warp per core row r in [r_begin, r_end): the row's columns in rounds
// of 32; lanes whose columns share a word OR their bits together
// (__match_any_sync + __reduce_or_sync) and the group's first lane writes
// the word. The warp is the row's only writer and its rounds are ordered
// by __syncwarp, so plain read-modify-writes suffice. Columns outside
// (v, v0 + h) are left out.
template <typename Off>
__global__ void k_core_bitmap(const Off *__restrict__ rp,
                              const uint32_t *__restrict__ ci, uint64_t v0,
                              uint32_t h, uint32_t H4, uint32_t *__restrict__ core,
                              uint32_t r_begin, uint32_t r_end) {
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t r = r_begin + warp; r < r_end; r += nwarps) {
    const uint64_t v = v0 + r;
    uint32_t *row = core + core_row_off(H4, (uint32_t)r) - core_row_first((uint32_t)r);
    const uint64_t e = ld_off(rp, v + 1);
    for (uint64_t j0 = ld_off(rp, v); j0 < e; j0 += 32) {
      const uint64_t j = j0 + lane;
      const uint64_t u = j < e ? (uint64_t)ci[j] : 0;
      const uint64_t c = u - v0;  // wraps for u < v0
      const bool ok = j < e && u > v && c < h;
      const uint32_t widx = ok ? (uint32_t)(c >> 5) : 0xFFFFFFFFu;
      const uint32_t peers = __match_any_sync(0xffffffffu, widx);
      const uint32_t bits = __reduce_or_sync(peers, ok ? 1u << (c & 31) : 0u);
      if (ok && lane == (uint32_t)__ffs(peers) - 1) row[widx] |= bits;
      __syncwarp();
    }
  }
}

// Sizing the dense core from the row offsets alone (before any column is
// needed): for each candidate length h_c (core_candidate(c), largest first),
// the wedges of the top h_c vertices and an estimate of the words their
// row ANDs read -- a pair (v, w) of local rows r_v < r_w reads the words
// from column r_w on, about (h_c - r_v) / 64 on average when w is spread
// over (r_v, h_c). out[2c] = wedges, out[2c + 1] = words; candidates
// core_candidate(c), largest first.
constexpr uint32_t kCoreNumCandidates = 9;
// Dense core sizing: at most kCoreMaxLen vertices (the core kernel's
// shared bit row is kCoreMaxH4 words). A candidate is eligible when it
// holds at least kCoreMinWedges wedges and its row ANDs read at most
// kCoreWordsPerWedge words per wedge they replace; the automatic size is
// the eligible candidate of least estimated time (core_pick).
constexpr uint64_t kCoreMaxLen = 32ull * kCoreMaxH4;
constexpr unsigned long long kCoreWordsPerWedge = 2;
constexpr unsigned long long kCoreMinWedges = 1ull << 22;
// A word read by the row ANDs costs about this fraction of a wedge check
// moved into the core (R-MAT scale 22 on B200, between neighbouring
// candidates from 8,192 to 65,536 vertices: 0.21 ps per estimated word,
// 2.0-2.7 ps per wedge moved out of the wedge-check kernel).
constexpr double kCoreWordsPerCheck = 8.0;
__host__ __device__ constexpr uint32_t core_candidate(uint32_t c) {
  // 65536, 57344, 49152, 40960, 32768, 16384, 8192, 4096, 2048
  return c < 5 ? 65536u - 8192u * c : 32768u >> (c - 4);
}
template <typename Off>
__global__ void k_core_plan(const Off *__restrict__ rp, uint64_t n,
                            unsigned long long *__restrict__ out) {
  unsigned long long acc[2 * kCoreNumCandidates] = {};
  const uint64_t top = n < core_candidate(0) ? n : core_candidate(0);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < top;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t v = n - top + i;
    const uint64_t d = ld_off(rp, v + 1) - ld_off(rp, v);
    const uint64_t wedges = d >= 2 ? d * (d - 1) / 2 : 0;
#pragma unroll
    for (uint32_t c = 0; c < kCoreNumCandidates; ++c) {
      const uint64_t hc = n < core_candidate(c) ? n : core_candidate(c);
      if (v >= n - hc) {
        acc[2 * c] += wedges;
        acc[2 * c + 1] += d * (hc - (v - (n - hc))) / 64 + d;
      }
    }
  }
#pragma unroll
  for (uint32_t c = 0; c < 2 * kCoreNumCandidates; ++c) {
    unsigned long long x = acc[c];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(out + c, x);
  }
}

// The automatic core from k_core_plan's read-back (plan[2c] = wedges,
// plan[2c + 1] = words of candidate c): among the eligible candidates, the
// least words - kCoreWordsPerCheck * wedges (the row ANDs' reads against
// the wedge checks they save); -1 = no core. Candidates that n caps to the
// same length tie, and the first of them is kept.
inline int core_pick(const unsigned long long *plan) {
  int pick = -1;
  double best = 0.0;
  for (uint32_t c = 0; c < kCoreNumCandidates; ++c) {
    const unsigned long long wedges = plan[2 * c], words = plan[2 * c + 1];
    if (wedges < kCoreMinWedges || words > kCoreWordsPerWedge * wedges) continue;
    const double score = (double)words - kCoreWordsPerCheck * (double)wedges;
    if (pick < 0 || score < best) {
      pick = (int)c;
      best = score;
    }
  }
  return pick;
}

// For each candidate first core vertex v0[i]: out[2i] = its active index
// (pos[v0]), out[2i + 1] = the wedge prefix there (the first core wedge).
struct CoreStarts {
  uint64_t v0[2 * kCoreNumCandidates + 2];
  uint32_t c;
};
__global__ void k_core_prefix(const uint64_t *__restrict__ act_wp,
                              const uint64_t *__restrict__ pos, CoreStarts cs,
                              uint64_t *__restrict__ out) {
  const uint32_t i = threadIdx.x;
  if (i < cs.c) {
    const uint64_t k = pos[cs.v0[i]];
    out[2 * i] = k;
    out[2 * i + 1] = act_wp[k];
  }
}

// Staging of one adjacency row N+(v) into shared memory by a TMA bulk copy
// (cp.async.bulk, one CTA, no multicast), completed on an mbarrier: the
// 16-byte-aligned body [rb & ~3, (rb + d) & ~3) goes by TMA, the ragged
// tail (< 4 columns) by plain loads; the row starts at stage[rb & 3]. Only
// when the column array is 16-byte aligned (tma_ok, checked by the host)
// and the row fits kStageCols columns; otherwise the caller reads global
// memory. The wait is bounded: on running out it records kDevStageTimeout
// in *err, waits once more (bounded) for the copy it started, and returns
// false.
constexpr uint32_t kStageCols = 2048;
constexpr uint32_t kStageSpin = 1u << 22;
constexpr uint32_t kDevStageTimeout = 6;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint32_t limit) {
  uint32_t done = 0;
  for (uint32_t it = 0; it < limit && !done; ++it)
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;"
        " selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
  return done != 0;
}

// All threads of the block call it; returns whether stage[] holds the row
// (at stage + (rb & 3)). mbar must be a fresh __shared__ u64 per call site.
__device__ __forceinline__ bool stage_row(const uint32_t *__restrict__ ci, uint64_t rb,
                                          uint32_t d, bool tma_ok, uint32_t *stage,
                                          unsigned long long *mbar_p, uint32_t *err) {
  const uint64_t a0 = rb & ~3ull, a1 = (rb + d) & ~3ull;
  const bool use = tma_ok && d >= 32 && a1 > a0 && (rb + d - a0) <= kStageCols;
  if (!use) return false;  // block-uniform
  const uint32_t mbar = smem_addr(mbar_p);
  const uint32_t bytes = (uint32_t)((a1 - a0) * 4);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar),
                 "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(stage)),
        "l"(ci + a0), "r"(bytes), "r"(mbar)
        : "memory");
  }
  // the tail by plain loads (columns [a1, rb + d))
  for (uint64_t j = a1 + threadIdx.x; j < rb + d; j += blockDim.x) stage[j - a0] = __ldg(ci + j);
  const bool ok = mbar_wait(mbar, 0, kStageSpin);
  if (!ok) {
    if (threadIdx.x == 0 && err) atomicCAS(err, 0u, kDevStageTimeout);
    mbar_wait(mbar, 0, kStageSpin);  // the copy this block started, once more
  }
  __syncthreads();
  return __syncthreads_and(ok ? 1 : 0) != 0;
}

// The first wedge of the pair (v, N+(v)[wi]) in the count's wedge order,
// P being v's first: the pairs before it hold (d-1) + (d-2) + ... wedges.
__device__ __forceinline__ uint64_t pair_first_wedge(uint64_t P, uint32_t d, uint32_t wi) {
  return P + (uint64_t)wi * (d - 1) - (uint64_t)wi * (wi ? wi - 1 : 0) / 2;
}

// Popcount of a & b over the columns [cmin, cmax) of word column jj.
__device__ __forceinline__ uint32_t masked_popc(uint32_t x, uint32_t jj,
                                                uint32_t cmin, uint32_t cmax) {
  const uint32_t lo = jj << 5;
  uint32_t m = 0xFFFFFFFFu;
  if (cmin > lo) m = cmin >= lo + 32 ? 0u : m << (cmin - lo);
  if (cmax < lo + 32) m &= cmax <= lo ? 0u : (0xFFFFFFFFu >> (lo + 32 - cmax));
  return __popc(x & m);
}

// One block per active core vertex (active entries [Kc, K), in order): the
// block builds its vertex's bit row in shared memory from N+(v), then each
// warp takes every 8th pair (v, w = N+(v)[wi]), 32 at a time, and ANDs the
// shared row with the core row of w, 16 bytes per lane. Only wedges in
// [lo, hi) are counted: a vertex or a pair outside it is skipped, and a
// pair the range cuts is masked to the columns of its counted wedges. One
// 64-bit atomic per block. Built for 8 blocks per SM (32 registers, 64
// warps): the row loads mostly hit L2 and more warps in flight hide their
// latency (R-MAT scale 22, core of 32,768, before the strided pairs: 1.55
// ms at 8 blocks per SM, 1.86 ms at 6).
template <typename Off>
__global__ void __launch_bounds__(kCoreBlock, 8)
    k_core_count(const uint32_t *__restrict__ ci,
                 const uint32_t *__restrict__ core, uint64_t v0, uint32_t h,
                 uint32_t H4, const uint64_t *__restrict__ act_wp,
                 const uint64_t *__restrict__ act_rb,
                 const uint32_t *__restrict__ act_d, uint64_t Kc, uint64_t K,
                 uint64_t lo, uint64_t hi, unsigned long long *__restrict__ out,
                 bool tma_ok = false, uint32_t *err = nullptr) {
  __shared__ __align__(16) uint32_t rv[kCoreMaxH4];
  __shared__ __align__(128) uint32_t stage[kStageCols];
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ unsigned long long warp_acc[kCoreBlock / 32];
  const uint64_t k = Kc + blockIdx.x;
  if (k >= K) return;
  const uint64_t P = __ldg(act_wp + k);
  const uint32_t d = __ldg(act_d + k);
  const uint64_t Wv = (uint64_t)d * (d - 1) / 2;
  if (P + Wv <= lo || P >= hi) return;  // block-uniform
  const uint64_t rb = __ldg(act_rb + k);
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (uint32_t i = tid; i < H4; i += kCoreBlock) rv[i] = 0;
  // N+(v), read twice below: staged in shared memory when it fits
  const bool staged = stage_row(ci, rb, d, tma_ok, stage, &mbar, err);
  const uint32_t *row_v = staged ? stage + (rb & 3) : ci + rb;
  __syncthreads();
  for (uint32_t j = tid; j < d; j += kCoreBlock) {
    const uint64_t c = (uint64_t)(staged ? row_v[j] : __ldg(row_v + j)) - v0;
    if (c < h) atomicOr(&rv[c >> 5], 1u << (c & 31));
  }
  __syncthreads();
  const bool whole = P >= lo && P + Wv <= hi;
  uint32_t acc = 0;
  // Warp q takes the pairs wi = q, q + 8, q + 16, ...: the rows of w get
  // shorter as wi grows (w's stored row starts at its own column), so
  // strided pairs give the block's warps equal work, where runs of 32
  // consecutive pairs left the first warps with the longest rows.
  constexpr uint32_t kWarps = kCoreBlock / 32;
  for (uint32_t base = warp; base + 1 < d; base += kCoreBlock) {
    // Lane p sets up the pair wi = base + kWarps * p once for the warp: the
    // first stored word j0 and the word offset of w's core row (below 2^27:
    // h <= 65536 rows of at most 2048 words), and whether the range cuts
    // it. A skipped pair keeps j0 = H4 (no words to AND).
    const uint32_t wl = base + kWarps * lane;
    uint32_t my_j0 = H4, my_off = 0;
    bool my_cut = false;
    if (wl + 1 < d) {
      const uint64_t cw = (uint64_t)(staged ? row_v[wl] : __ldg(row_v + wl)) - v0;
      bool on = cw < h;  // else not a core column (invalid input)
      if (on && !whole) {
        const uint64_t ps = pair_first_wedge(P, d, wl), pl = d - 1 - wl;
        if (ps + pl <= lo || ps >= hi)
          on = false;
        else
          my_cut = ps < lo || ps + pl > hi;
      }
      if (on) {
        my_j0 = core_row_first((uint32_t)cw);
        my_off = (uint32_t)core_row_off(H4, (uint32_t)cw);
      }
    }
    const uint32_t cuts = __ballot_sync(0xffffffffu, my_cut);
    const uint32_t cnt = __popc(__ballot_sync(0xffffffffu, wl + 1 < d));
    for (uint32_t p = 0; p < cnt; ++p) {
      const uint32_t j0 = __shfl_sync(0xffffffffu, my_j0, p);
      const uint32_t off = __shfl_sync(0xffffffffu, my_off, p);
      const uint4 *row = reinterpret_cast<const uint4 *>(core + off);
      const uint4 *mine = reinterpret_cast<const uint4 *>(rv + j0);
      const uint32_t nq = (H4 - j0) >> 2;
      const bool cut = (cuts >> p) & 1u;
      if (!cut) {
        // not unrolled: the unrolled loop needs more than 32 registers
#pragma unroll 1
        for (uint32_t q = lane; q < nq; q += 32) {
          const uint4 a = __ldg(row + q);
          const uint4 b = mine[q];
          acc += __popc(a.x & b.x) + __popc(a.y & b.y) + __popc(a.z & b.z) +
                 __popc(a.w & b.w);
        }
      } else {
        // the counted columns of the pair wi: u indices [ulo, uhi)
        const uint32_t wi = base + kWarps * p;
        const uint64_t ps = pair_first_wedge(P, d, wi), pl = d - 1 - wi;
        const uint64_t ulo = wi + 1 + (ps < lo ? lo - ps : 0);
        const uint64_t uhi = wi + 1 + (ps + pl > hi ? hi - ps : pl);  // exclusive
        const uint32_t cmin = (uint32_t)((uint64_t)__ldg(ci + rb + ulo) - v0);
        const uint32_t cmax = (uint32_t)((uint64_t)__ldg(ci + rb + uhi - 1) - v0) + 1;
        for (uint32_t q = lane; q < nq; q += 32) {
          const uint4 a = __ldg(row + q);
          const uint4 b = mine[q];
          const uint32_t jj = j0 + 4 * q;
          acc += masked_popc(a.x & b.x, jj, cmin, cmax) +
                 masked_popc(a.y & b.y, jj + 1, cmin, cmax) +
                 masked_popc(a.z & b.z, jj + 2, cmin, cmax) +
                 masked_popc(a.w & b.w, jj + 3, cmin, cmax);
        }
      }
    }
  }
  const uint32_t tot = __reduce_add_sync(0xffffffffu, acc);
  if (lane == 0) warp_acc[warp] = tot;
  __syncthreads();
  if (tid == 0) {
    unsigned long long t = 0;
    for (uint32_t q = 0; q < kCoreBlock / 32; ++q) t += warp_acc[q];
    if (t) atomicAdd(out, t);
  }
}

// The shell: the vertices just below the core, [v1, v0), one block each.
// Their out-neighbours straddle the core boundary, so each pair (v, w) is
// counted the cheaper way: for w in the core, a row AND of v's core bits
// (built in shared memory) with w's core row when that reads no more
// 16-byte words than the pair has wedges, else bit tests of the pair's
// columns in w's core row; for w below the core, the wedge checks of the
// count kernel (segment_hits: near set, hash set or search). The core
// matrix is the count's bitmap here (aligned mode). Wedge ranges are exact
// as in k_core_count: a pair the range cuts counts only its columns
// [ulo, uhi).
template <typename Off, bool kNear>
__global__ void __launch_bounds__(kCoreBlock)
    k_shell_count(const Off *__restrict__ rp, const uint32_t *__restrict__ ci,
                  uint64_t n, const uint32_t *__restrict__ core, uint64_t v0,
                  uint32_t h, uint32_t H4, const uint64_t *__restrict__ act_wp,
                  const uint64_t *__restrict__ act_rb,
                  const uint32_t *__restrict__ act_d, uint64_t Ks, uint64_t Kc,
                  uint64_t lo, uint64_t hi, HashView hv,
                  unsigned long long *__restrict__ out, bool tma_ok = false,
                  uint32_t *err = nullptr) {
  __shared__ __align__(16) uint32_t rv[kCoreMaxH4];
  __shared__ __align__(128) uint32_t stage[kStageCols];
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ unsigned long long warp_acc[kCoreBlock / 32];
  const uint64_t k = Ks + blockIdx.x;
  if (k >= Kc) return;
  const uint64_t P = __ldg(act_wp + k);
  const uint32_t d = __ldg(act_d + k);
  const uint64_t Wv = (uint64_t)d * (d - 1) / 2;
  if (P + Wv <= lo || P >= hi) return;  // block-uniform
  const uint64_t rb = __ldg(act_rb + k);
  const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (uint32_t i = tid; i < H4; i += kCoreBlock) rv[i] = 0;
  // N+(v), read twice below: staged in shared memory when it fits
  const bool staged = stage_row(ci, rb, d, tma_ok, stage, &mbar, err);
  const uint32_t *row_v = staged ? stage + (rb & 3) : ci + rb;
  __syncthreads();
  for (uint32_t j = tid; j < d; j += kCoreBlock) {
    const uint64_t c = (uint64_t)(staged ? row_v[j] : __ldg(row_v + j)) - v0;
    if (c < h) atomicOr(&rv[c >> 5], 1u << (c & 31));
  }
  __syncthreads();
  const bool whole = P >= lo && P + Wv <= hi;
  uint32_t acc = 0;
  for (uint32_t base = warp * 32; base + 1 < d; base += kCoreBlock) {
    const uint32_t wl = base + lane;
    const uint32_t wcol = wl + 1 < d ? (staged ? row_v[wl] : __ldg(row_v + wl)) : 0u;
    const uint32_t cnt = d - 1 - base < 32 ? d - 1 - base : 32;
    for (uint32_t p = 0; p < cnt; ++p) {
      const uint32_t wi = base + p;
      const uint32_t w = __shfl_sync(0xffffffffu, wcol, p);
      // the pair's counted columns: u indices [ulo, uhi)
      uint32_t ulo = wi + 1, uhi = d;
      bool cut = false;
      if (!whole) {
        const uint64_t ps = P + (uint64_t)wi * (d - 1) - (uint64_t)wi * (wi ? wi - 1 : 0) / 2;
        const uint64_t pl = d - 1 - wi;
        if (ps + pl <= lo || ps >= hi) continue;
        if (ps < lo || ps + pl > hi) {
          cut = true;
          ulo = (uint32_t)(wi + 1 + (ps < lo ? lo - ps : 0));
          uhi = (uint32_t)(wi + 1 + (ps + pl > hi ? hi - ps : pl));
        }
      }
      const uint64_t cw = (uint64_t)w - v0;
      if (cw < h) {
        const uint32_t r = (uint32_t)cw;
        const uint32_t j0 = core_row_first(r);
        const uint32_t nq = (H4 - j0) >> 2;
        if (nq <= uhi - ulo) {
          const uint4 *row = reinterpret_cast<const uint4 *>(core + core_row_off(H4, r));
          const uint4 *mine = reinterpret_cast<const uint4 *>(rv + j0);
          if (!cut) {
            for (uint32_t q = lane; q < nq; q += 32) {
              const uint4 a = __ldg(row + q);
              const uint4 b = mine[q];
              acc += __popc(a.x & b.x) + __popc(a.y & b.y) + __popc(a.z & b.z) +
                     __popc(a.w & b.w);
            }
          } else {
            const uint32_t cmin = (uint32_t)((uint64_t)__ldg(ci + rb + ulo) - v0);
            const uint32_t cmax = (uint32_t)((uint64_t)__ldg(ci + rb + uhi - 1) - v0) + 1;
            for (uint32_t q = lane; q < nq; q += 32) {
              const uint4 a = __ldg(row + q);
              const uint4 b = mine[q];
              const uint32_t jj = j0 + 4 * q;
              acc += masked_popc(a.x & b.x, jj, cmin, cmax) +
                     masked_popc(a.y & b.y, jj + 1, cmin, cmax) +
                     masked_popc(a.z & b.z, jj + 2, cmin, cmax) +
                     masked_popc(a.w & b.w, jj + 3, cmin, cmax);
            }
          }
          continue;
        }
      }
      acc += segment_hits<Off, false, true, kNear, true>(rp, ci, n, core, v0, H4, BatchView{}, 0,
                                                         hv, w, ci + rb + ulo, uhi - ulo);
    }
  }
  const uint32_t tot = __reduce_add_sync(0xffffffffu, acc);
  if (lane == 0) warp_acc[warp] = tot;
  __syncthreads();
  if (tid == 0) {
    unsigned long long t = 0;
    for (uint32_t q = 0; q < kCoreBlock / 32; ++q) t += warp_acc[q];
    if (t) atomicAdd(out, t);
  }
}

// Per oriented entry (v, position p): the (d+(v) - p - 1) wedges with
// middle vertex w = ci[p] each cost 4 + 16 + 4*ceil(log2(d+(w) + 1)) bytes.
template <typename Off>
__global__ void k_alg_bytes(const Off *__restrict__ rp,
                            const uint32_t *__restrict__ ci, uint64_t n,
                            uint64_t m, unsigned long long *out) {
  const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long acc = 0;
  for (uint64_t v = warp; v < n; v += nwarps) {
    const uint64_t b = ld_off(rp, v), e = ld_off(rp, v + 1);
    if (e < b || e > m) continue;
    for (uint64_t j = b + lane; j < e; j += 32) {
      const uint64_t wedges = e - j - 1;
      if (wedges == 0) continue;
      const uint64_t w = ci[j];
      const uint64_t wb = w < n ? ld_off(rp, w) : 0;
      const uint64_t we = w < n ? ld_off(rp, w + 1) : 0;
      const uint64_t dw = we > wb ? we - wb : 0;
      // ceil(log2(dw + 1)) = bit length of dw
      const uint64_t probes = dw == 0 ? 0 : 64 - __clzll((long long)dw);
      acc += wedges * (4 + 16 + 4 * probes);
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0 && acc) atomicAdd(out, acc);
}

__global__ void k_narrow(const uint64_t *__restrict__ a, uint64_t n,
                         uint32_t *__restrict__ b) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n;
       i += (uint64_t)gridDim.x * blockDim.x)
    b[i] = (uint32_t)a[i];
}

__global__ void k_widen(const uint32_t *__restrict__ a, uint64_t n,
                        uint64_t *__restrict__ b) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n;
       i += (uint64_t)gridDim.x * blockDim.x)
    b[i] = a[i];
}

}  // namespace
}  // namespace wetric
