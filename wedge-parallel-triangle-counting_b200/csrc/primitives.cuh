// primitives.cuh -- device-wide exclusive scan and stable LSD radix sort,
// written for this library in place of the CUB calls of the reference
// (DeviceRadixSort / DeviceSegmentedSort, tc.cu:500-558).
//
// Neither primitive waits on another block: the scan is reduce-then-scan
// (three launches) and the sort is histogram / scan / scatter per digit,
// so no kernel here can spin.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace wetric {
namespace prim {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanChunk = kScanThreads * kScanItems;

// Inclusive scan of one value per thread across a 256-thread block.
// Returns the inclusive prefix; *total receives the block total.
template <typename T>
__device__ __forceinline__ T block_inclusive_scan(T v, T *smem_warp, T *total) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += y;
  }
  if (lane == 31) smem_warp[warp] = v;
  __syncthreads();
  if (warp == 0) {
    T w = lane < (kScanThreads / 32) ? smem_warp[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < (kScanThreads / 32)) smem_warp[lane] = w;
  }
  __syncthreads();
  if (warp > 0) v += smem_warp[warp - 1];
  *total = smem_warp[kScanThreads / 32 - 1];
  return v;
}

template <typename InT, typename OutT>
__global__ void __launch_bounds__(kScanThreads)
    scan_reduce_kernel(const InT *__restrict__ in, uint64_t n,
                       OutT *__restrict__ block_sums) {
  __shared__ OutT warp_sums[kScanThreads / 32];
  const uint64_t base =
      (uint64_t)blockIdx.x * kScanChunk + (uint64_t)threadIdx.x * kScanItems;
  OutT s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    const uint64_t i = base + j;
    if (i < n) s += (OutT)in[i];
  }
  OutT total;
  block_inclusive_scan<OutT>(s, warp_sums, &total);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

// out[i] = offset(block) + exclusive prefix within the block. When
// block_offsets is null the offset is 0. The block that owns element n-1
// (or block 0 when n == 0) also writes out[n] = total.
template <typename InT, typename OutT>
__global__ void __launch_bounds__(kScanThreads)
    scan_apply_kernel(const InT *in, uint64_t n, OutT *out,
                      const OutT *__restrict__ block_offsets) {
  __shared__ OutT warp_sums[kScanThreads / 32];
  const uint64_t base =
      (uint64_t)blockIdx.x * kScanChunk + (uint64_t)threadIdx.x * kScanItems;
  OutT vals[kScanItems];
  OutT s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    const uint64_t i = base + j;
    vals[j] = i < n ? (OutT)in[i] : OutT(0);
    s += vals[j];
  }
  OutT total;
  OutT incl = block_inclusive_scan<OutT>(s, warp_sums, &total);
  OutT run = incl - s + (block_offsets ? block_offsets[blockIdx.x] : OutT(0));
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    const uint64_t i = base + j;
    if (i < n) out[i] = run;
    run += vals[j];
  }
  const uint64_t block_end = (uint64_t)(blockIdx.x + 1) * kScanChunk;
  if (threadIdx.x == kScanThreads - 1 && block_end >= n) {
    out[n] = (block_offsets ? block_offsets[blockIdx.x] : OutT(0)) + total;
  }
}

// out[0..n] = exclusive prefix of in[0..n-1]; out[n] = total. out may alias
// in when InT == OutT.
template <typename InT, typename OutT>
int exclusive_scan(DeviceContext *ctx, cudaStream_t st, const InT *in,
                   OutT *out, uint64_t n) {
  const uint64_t blocks = n == 0 ? 1 : ceil_div(n, kScanChunk);
  if (blocks == 1) {
    scan_apply_kernel<InT, OutT><<<1, kScanThreads, 0, st>>>(in, n, out,
                                                             nullptr);
    WETRIC_LAUNCH_CHECK();
    return WETRIC_OK;
  }
  Scratch<OutT> sums;
  WETRIC_TRY(sums.alloc(ctx, st, blocks + 1));
  scan_reduce_kernel<InT, OutT><<<(unsigned)blocks, kScanThreads, 0, st>>>(
      in, n, sums.ptr);
  WETRIC_LAUNCH_CHECK();
  WETRIC_TRY((exclusive_scan<OutT, OutT>(ctx, st, sums.ptr, sums.ptr, blocks)));
  scan_apply_kernel<InT, OutT><<<(unsigned)blocks, kScanThreads, 0, st>>>(
      in, n, out, sums.ptr);
  WETRIC_LAUNCH_CHECK();
  return WETRIC_OK;
}

// ------------------------------------------------------------ radix sort

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 8;  // per lane
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;

// Tile layout (shared by the histogram and scatter kernels, which is what
// keeps the sort stable): warp w of tile t owns the contiguous keys
// [t*Tile + w*32*Items, +32*Items); item j of lane l is key
// [that base + j*32 + l], so every load is coalesced and the order
// (warp, item, lane) is the input order.
template <typename K>
__global__ void __launch_bounds__(kSortThreads)
    radix_hist_kernel(const K *__restrict__ keys, uint64_t n, uint32_t shift,
                      uint64_t num_tiles, uint32_t *__restrict__ counts) {
  __shared__ uint32_t hist[kRadix];
  for (int d = threadIdx.x; d < kRadix; d += kSortThreads) hist[d] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const uint64_t sub = (uint64_t)blockIdx.x * kSortTile +
                       (uint64_t)warp * 32 * kSortItems;
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const uint64_t i = sub + (uint64_t)j * 32 + lane;
    if (i < n) {
      const uint32_t d = (uint32_t)(keys[i] >> shift) & (kRadix - 1);
      atomicAdd(&hist[d], 1u);
    }
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadix; d += kSortThreads)
    counts[(uint64_t)d * num_tiles + blockIdx.x] = hist[d];
}

template <typename K, typename V, bool kHasValues>
__global__ void __launch_bounds__(kSortThreads)
    radix_scatter_kernel(const K *__restrict__ keys_in,
                         const V *__restrict__ vals_in, uint64_t n,
                         uint32_t shift, uint64_t num_tiles,
                         const uint64_t *__restrict__ offsets,
                         K *__restrict__ keys_out, V *__restrict__ vals_out) {
  __shared__ uint32_t whist[kSortWarps][kRadix];
  __shared__ uint64_t goff[kRadix];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  for (int d = threadIdx.x; d < kRadix; d += kSortThreads) {
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) whist[w][d] = 0;
    goff[d] = offsets[(uint64_t)d * num_tiles + blockIdx.x];
  }
  __syncthreads();

  const uint64_t sub = (uint64_t)blockIdx.x * kSortTile +
                       (uint64_t)warp * 32 * kSortItems;
  const uint32_t lt_mask = (1u << lane) - 1u;
  K k[kSortItems];
  V v[kSortItems];
  uint32_t rank[kSortItems];
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const uint64_t i = sub + (uint64_t)j * 32 + lane;
    const bool valid = i < n;
    k[j] = valid ? keys_in[i] : K(0);
    if (kHasValues) v[j] = valid ? vals_in[i] : V(0);
    const uint32_t d = (uint32_t)(k[j] >> shift) & (kRadix - 1);
    const uint32_t tag = valid ? d : 0xFFFFFFFFu;
    const uint32_t peers = __match_any_sync(0xffffffffu, tag);
    uint32_t before = 0;
    if (valid) before = whist[warp][d];
    __syncwarp();
    if (valid && lane == __ffs(peers) - 1) whist[warp][d] = before + __popc(peers);
    __syncwarp();
    rank[j] = before + __popc(peers & lt_mask);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadix; d += kSortThreads) {
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t c = whist[w][d];
      whist[w][d] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    const uint64_t i = sub + (uint64_t)j * 32 + lane;
    if (i < n) {
      const uint32_t d = (uint32_t)(k[j] >> shift) & (kRadix - 1);
      const uint64_t pos = goff[d] + whist[warp][d] + rank[j];
      keys_out[pos] = k[j];
      if (kHasValues) vals_out[pos] = v[j];
    }
  }
}

// Stable LSD sort of keys (and optional values) on their low `bits` bits.
// Ping-pongs between (keys, keys_alt); *result_in_alt tells which buffer
// holds the sorted output.
template <typename K, typename V>
int radix_sort(DeviceContext *ctx, cudaStream_t st, K *keys, K *keys_alt,
               V *vals, V *vals_alt, uint64_t n, uint32_t bits,
               bool *result_in_alt) {
  *result_in_alt = false;
  if (n <= 1 || bits == 0) return WETRIC_OK;
  const uint64_t num_tiles = ceil_div(n, kSortTile);
  const uint64_t ncounts = (uint64_t)kRadix * num_tiles;
  Scratch<uint32_t> counts;
  Scratch<uint64_t> offsets;
  WETRIC_TRY(counts.alloc(ctx, st, ncounts));
  WETRIC_TRY(offsets.alloc(ctx, st, ncounts + 1));
  K *kin = keys, *kout = keys_alt;
  V *vin = vals, *vout = vals_alt;
  bool in_alt = false;
  for (uint32_t shift = 0; shift < bits; shift += kRadixBits) {
    radix_hist_kernel<K><<<(unsigned)num_tiles, kSortThreads, 0, st>>>(
        kin, n, shift, num_tiles, counts.ptr);
    WETRIC_LAUNCH_CHECK();
    WETRIC_TRY((exclusive_scan<uint32_t, uint64_t>(ctx, st, counts.ptr,
                                                   offsets.ptr, ncounts)));
    if (vals != nullptr) {
      radix_scatter_kernel<K, V, true>
          <<<(unsigned)num_tiles, kSortThreads, 0, st>>>(
              kin, vin, n, shift, num_tiles, offsets.ptr, kout, vout);
    } else {
      radix_scatter_kernel<K, V, false>
          <<<(unsigned)num_tiles, kSortThreads, 0, st>>>(
              kin, vin, n, shift, num_tiles, offsets.ptr, kout, vout);
    }
    WETRIC_LAUNCH_CHECK();
    K *tk = kin; kin = kout; kout = tk;
    V *tv = vin; vin = vout; vout = tv;
    in_alt = !in_alt;
  }
  *result_in_alt = in_alt;
  return WETRIC_OK;
}

}  // namespace prim
}  // namespace wetric
