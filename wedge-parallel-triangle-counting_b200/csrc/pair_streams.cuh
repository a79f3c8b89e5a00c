// pair_streams.cuh -- the count of short rows by pair streams.
//
// The wedge check (tc.cu:252-287) reads one set of a middle vertex per
// wedge: a random bucket of u's set for the wedge (v; u, w). On graphs
// without hubs (Erdos-Renyi, mild power laws) nearly every row is short and
// those reads are what the count spends its time on: about 7 warp
// instructions per wedge in the per-lane rounds of the row walk. A pair
// stream counts the same triangles the other way round: for a short row v
// (d+(v) <= 64) the warp builds a set of N+(v) in shared memory and, for
// every pair (v, u) with u in N+(v), streams the columns x of N+(u) through
// it; x in N+(v) closes the triangle (v, u, x), and since every x of N+(u)
// is above u, the hits of (v, u) are exactly the triangles of the wedges
// (v; u, w), w > u, that the wedge check would find -- so a vertex's count
// is the same either way. The columns come in coalesced, 32 per round, the
// lookups are shared-memory loads, and the rounds pack the streams of
// consecutive pairs (a warp-wide search maps each lane's position to its
// pair), so no lane idles between short rows.
//
// A vertex takes the pair stream when that is cheaper by a cost model in
// warp instructions (setup per vertex plus one round per 32 streamed
// columns, against the wedge check's per-wedge cost: high in the per-lane
// rounds of short row tails, low in whole-warp segment rounds); the
// rest, and every wedge of a vertex with d+ > 64, stay with the wedge
// check. The split is by whole vertices, so it changes no count.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "count_kernels.cuh"

namespace wetric {
namespace {

constexpr uint32_t kPairMaxDeg = 64;        // rows with d+ <= 64
constexpr uint32_t kPairSlots = 128;        // set of N+(v): load <= 1/2
constexpr uint32_t kPairEmpty = 0xFFFFFFFFu;
constexpr uint32_t kPairWarps = 8;          // warps per block
// Cost model, warp instructions: a pair-stream vertex costs about
// kPairVertexCost to set up and kPairRoundCost per round of 32 columns;
// the wedge check costs about kPairWedgeCost per wedge whose row tail is
// shorter than a segment (kPairSegMin wedges: per-lane rounds) and
// kPairSegWedgeCost per wedge of a longer tail (whole-warp segment
// rounds). On the uneven 4,096-graph mixture this split measured 5,895
// graphs/s against 5,352 with every wedge at 7 and 5,627 at 4, and a setup
// cost of 160 5,996 against 5,971 at 80 and 5,915 at 40.
constexpr uint32_t kPairVertexCost = 160;
constexpr uint32_t kPairRoundCost = 30;
constexpr uint32_t kPairWedgeCost = 7;
constexpr uint32_t kPairSegWedgeCost = 2;
constexpr uint32_t kPairSegMin = 16;
constexpr uint32_t kPairTile = 2048;        // streamed columns per warp tile
// Single-graph counts of fewer columns do not plan pair streams: the plan's
// launches would cost more than the streams save.
constexpr uint64_t kPairMinColumns = 1u << 15;

// Columns per pair-stream tile for R streamed columns on a device of
// `sms` SMs: kPairTile, or fewer (whole rounds, at least 256) when that
// leaves fewer than about two tiles per warp slot of the device.
inline uint64_t pair_tile_cols(uint64_t R, int sms) {
  uint64_t T = kPairTile;
  const uint64_t min_tiles = 2ull * (uint64_t)sms * 64;
  if (ceil_div(R, T) < min_tiles) {
    const uint64_t t = ceil_div(ceil_div(R, min_tiles), 32) * 32;
    T = t < T ? (t < 256 ? 256 : t) : T;
  }
  return T;
}

__device__ __forceinline__ uint32_t pair_slot(uint32_t x) {
  return (x * 0x9E3779B1u) >> 25;  // top 7 bits: kPairSlots = 128
}

// Streamed-column budget of a vertex with d out-neighbours: the largest R
// for which its pair streams are cheaper than its wedge checks (0: never).
// Row tails of a vertex with d columns: d - 1, d - 2, ..., 1 wedges; the
// tails below kPairSegMin hold S = t(t+1)/2 wedges (t = min(d-1, 15)).
__host__ __device__ __forceinline__ uint64_t pair_budget(uint64_t d) {
  if (d < 2 || d > kPairMaxDeg) return 0;
  const uint64_t t = d - 1 < kPairSegMin - 1 ? d - 1 : kPairSegMin - 1;
  const uint64_t short_w = t * (t + 1) / 2, all_w = d * (d - 1) / 2;
  const uint64_t wedge_cost =
      (uint64_t)kPairWedgeCost * short_w + (uint64_t)kPairSegWedgeCost * (all_w - short_w);
  if (wedge_cost <= kPairVertexCost) return 0;
  return (wedge_cost - kPairVertexCost) * 32 / kPairRoundCost;
}

// Which vertices below v_end take pair streams: each one leaves the active
// set (the wedge check skips it) and is appended to pv with its stream
// length R(v) in pl -- the sum of d+(u) over u in N+(v) but its last column
// (whose pair has no wedges) -- by one atomic per warp; acc[0] counts them,
// acc[1] sums their wedges and acc[2] their R. Rows whose R passes the
// budget stop reading early. The order of pv is arbitrary (the count is a
// sum over it). kOrdered instead writes per vertex -- pv[v] = 1 for a pair
// vertex, pl[v] = R(v) -- for a scan to put them in vertex order
// (k_pair_compact), which a batch wants so that a tile stays in one graph.
template <bool kOrdered = false>
__global__ void k_pair_plan(const uint32_t *__restrict__ rp,
                            const uint32_t *__restrict__ ci, uint64_t v_end,
                            uint32_t *__restrict__ active,
                            uint32_t *__restrict__ pv, uint32_t *__restrict__ pl,
                            unsigned long long *__restrict__ acc) {
  const uint32_t lane = threadIdx.x & 31;
  unsigned long long wsum = 0, rsum = 0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  // whole warps step together, so the ballot sees every lane
  for (uint64_t v0 = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); v0 < v_end;
       v0 += stride) {
    const uint64_t v = v0 + lane;
    bool flag = false;
    uint32_t R = 0;
    if (v < v_end && active[v]) {
      const uint32_t b = rp[v], d = rp[v + 1] - b;
      const uint64_t budget = pair_budget(d);
      if (budget) {
        uint64_t r = 0;
        for (uint32_t j = 0; j + 1 < d && r <= budget; ++j) {
          const uint32_t u = __ldg(ci + b + j);
          r += __ldg(rp + u + 1) - __ldg(rp + u);
        }
        if (r <= budget) {
          flag = true;
          R = (uint32_t)r;
          active[v] = 0;
          wsum += (uint64_t)d * (d - 1) / 2;
          rsum += r;
        }
      }
    }
    if (kOrdered) {
      if (v < v_end) {
        pv[v] = flag ? 1u : 0u;
        pl[v] = R;
      }
      continue;
    }
    const uint32_t mask = __ballot_sync(0xffffffffu, flag);
    if (mask) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(acc, (unsigned long long)__popc(mask));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (flag) {
        const uint64_t k = base + __popc(mask & ((1u << lane) - 1u));
        pv[k] = (uint32_t)v;
        pl[k] = R;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    wsum += __shfl_down_sync(0xffffffffu, wsum, o);
    rsum += __shfl_down_sync(0xffffffffu, rsum, o);
  }
  if (lane == 0 && wsum) {
    atomicAdd(acc + 1, wsum);
    atomicAdd(acc + 2, rsum);
  }
}

// The pair vertices in vertex order (after k_pair_plan<true> and a scan of
// its flags into pos): out_v[k] = v, out_l[k] = R(v).
__global__ void k_pair_compact(const uint32_t *__restrict__ is_pair, uint64_t n,
                               const uint64_t *__restrict__ pos,
                               const uint32_t *__restrict__ len,
                               uint32_t *__restrict__ out_v, uint32_t *__restrict__ out_l) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x)
    if (is_pair[v]) {
      const uint64_t k = pos[v];
      out_v[k] = (uint32_t)v;
      out_l[k] = len[v];
    }
}

__device__ __forceinline__ void pair_insert(uint32_t *set, uint32_t u) {
  uint32_t h = pair_slot(u);
  for (;;) {
    const uint32_t old = atomicCAS(set + h, kPairEmpty, u);
    if (old == kPairEmpty || old == u) return;
    h = (h + 1) & (kPairSlots - 1);
  }
}

__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t x, uint32_t lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  return x;
}

// One warp per tile of kPairTile (or T) streamed columns over the
// pair-stream vertices' concatenated streams (ps: exclusive prefix of R,
// Kp + 1 entries; tile_k[t]: the vertex holding the tile's first column).
// kBatch: hits go to counts[pg[k]] (the vertex's graph), else to *total.
template <bool kBatch>
__global__ void __launch_bounds__(kPairWarps * 32, 8)
    k_count_pairs(const uint32_t *__restrict__ rp, const uint32_t *__restrict__ ci,
                  const uint32_t *__restrict__ pv, const uint64_t *__restrict__ ps,
                  const uint32_t *__restrict__ pg, uint64_t Kp,
                  const uint32_t *__restrict__ tile_k, uint64_t tiles, uint64_t T,
                  unsigned long long *__restrict__ total,
                  unsigned long long *__restrict__ counts) {
  __shared__ uint32_t s_set[kPairWarps][kPairSlots];
  // entry e: column index of its stream position 0 (row start minus stream
  // start, mod 2^32: position q reads column s_off[e] + q) and its start
  __shared__ uint32_t s_off[kPairWarps][kPairMaxDeg];
  __shared__ uint32_t s_start[kPairWarps][kPairMaxDeg];
  const uint32_t wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint64_t t = (uint64_t)blockIdx.x * kPairWarps + wid;
  if (t >= tiles) return;
  uint32_t *set = s_set[wid];
  uint32_t *eoff = s_off[wid];
  uint32_t *estart = s_start[wid];
  const uint64_t R = ps[Kp];
  const uint64_t tb = t * T;
  const uint64_t te = tb + T < R ? tb + T : R;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t le = 0xFFFFFFFFu >> (31 - lane);
  uint32_t hits = 0;
  uint32_t cur_g = 0;
  if (kBatch) cur_g = __ldg(pg + tile_k[t]);
  for (uint64_t k = tile_k[t]; k < Kp; ++k) {
    const uint64_t s0 = ps[k];
    if (s0 >= te) break;
    const uint64_t s1 = ps[k + 1];
    if (s1 <= tb || s1 == s0) continue;
    if (kBatch) {
      const uint32_t g = __ldg(pg + k);
      if (g != cur_g) {
        const uint32_t c = __reduce_add_sync(0xffffffffu, hits);
        if (lane == 0 && c) atomicAdd(counts + cur_g, (unsigned long long)c);
        hits = 0;
        cur_g = g;
      }
    }
    const uint32_t v = __ldg(pv + k);
    const uint32_t b = __ldg(rp + v), d = __ldg(rp + v + 1) - b;
#pragma unroll
    for (uint32_t i = lane; i < kPairSlots; i += 32) set[i] = kPairEmpty;
    __syncwarp();
    // rows of up to 33 columns (most of them) have at most 32 entries: the
    // second half of the warp's registers is skipped (warp-uniform branch)
    const bool two = d > 33;
    const uint32_t u0 = lane < d ? __ldg(ci + b + lane) : 0u;
    const uint32_t u1 = lane + 32 < d ? __ldg(ci + b + 32 + lane) : 0u;
    if (lane < d) pair_insert(set, u0);
    if (lane + 32 < d) pair_insert(set, u1);
    // entries: the pairs (v, u_i), i < d - 1, with their stream lengths
    uint32_t r0 = 0, l0 = 0, r1 = 0, l1 = 0;
    if (lane + 1 < d) {
      r0 = __ldg(rp + u0);
      l0 = __ldg(rp + u0 + 1) - r0;
    }
    if (lane + 33 < d) {
      r1 = __ldg(rp + u1);
      l1 = __ldg(rp + u1 + 1) - r1;
    }
    const uint32_t i0 = warp_inclusive_scan(l0, lane);
    const uint32_t tot0 = two ? __shfl_sync(0xffffffffu, i0, 31) : 0u;
    const uint32_t i1 = two ? warp_inclusive_scan(l1, lane) : 0u;
    // the entries with columns, in order (their starts are distinct)
    const uint32_t m0 = __ballot_sync(0xffffffffu, l0 > 0);
    const uint32_t m1 = two ? __ballot_sync(0xffffffffu, l1 > 0) : 0u;
    if (l0) {
      const uint32_t p = __popc(m0 & lt);
      eoff[p] = r0 - (i0 - l0);
      estart[p] = i0 - l0;
    }
    if (l1) {
      const uint32_t p = __popc(m0) + __popc(m1 & lt);
      eoff[p] = r1 - (tot0 + i1 - l1);
      estart[p] = tot0 + i1 - l1;
    }
    const uint32_t ne = __popc(m0) + __popc(m1);
    __syncwarp();
    const uint32_t c0 = lane < ne ? estart[lane] : 0xFFFFFFFFu;
    const uint32_t c1 = two && lane + 32 < ne ? estart[lane + 32] : 0xFFFFFFFFu;
    const uint32_t q0 = tb > s0 ? (uint32_t)(tb - s0) : 0u;
    const uint32_t q1 = (uint32_t)((te < s1 ? te : s1) - s0);
    // entry of position q = the last entry starting at or before q: the
    // entries starting before the round (counted once, then carried) plus
    // those starting in it up to the lane
    uint32_t before = __popc(__ballot_sync(0xffffffffu, c0 < q0)) +
                      __popc(__ballot_sync(0xffffffffu, c1 < q0));
    for (uint32_t base = q0; base < q1; base += 32) {
      uint32_t bits = 0;
      if (c0 - base < 32u) bits |= 1u << (c0 - base);
      if (c1 - base < 32u) bits |= 1u << (c1 - base);
      const uint32_t starts = __reduce_or_sync(0xffffffffu, bits);
      const uint32_t q = base + lane;
      const uint32_t e = before + __popc(starts & le) - 1;
      before += __popc(starts);
      if (q < q1) {
        const uint32_t x = __ldg(ci + (eoff[e] + q));
        uint32_t h = pair_slot(x);
        for (;;) {
          const uint32_t key = set[h];
          if (key == x) {
            ++hits;
            break;
          }
          if (key == kPairEmpty) break;
          h = (h + 1) & (kPairSlots - 1);
        }
      }
    }
    __syncwarp();
  }
  const uint32_t c = __reduce_add_sync(0xffffffffu, hits);
  if (lane == 0 && c) {
    if (kBatch)
      atomicAdd(counts + cur_g, (unsigned long long)c);
    else
      atomicAdd(total, (unsigned long long)c);
  }
}

}  // namespace
}  // namespace wetric
