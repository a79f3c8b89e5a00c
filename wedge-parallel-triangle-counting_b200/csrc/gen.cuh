// gen.cuh -- seeded synthetic graph streams, identical on host and device.
//
// The reference ships no generator (it reads files only, tc.cu:561); these
// produce the synthetic inputs that stand in for its datasets. Every draw is
// a pure function of (seed, counter) -- the splitmix64 output function
// (Steele, Lea, Flood, "Fast splittable pseudorandom number generators",
// OOPSLA 2014) applied to seed + (i + 1) * golden-gamma -- and every
// probability is compared in integer arithmetic, so a host loop and a CUDA
// kernel produce the same edge stream bit for bit.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define WETRIC_HD __host__ __device__ __forceinline__
#else
#define WETRIC_HD inline
#endif

namespace wetric {
namespace gen {

constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ull;

// i-th output of a splitmix64 generator seeded with `seed`.
WETRIC_HD uint64_t splitmix64_at(uint64_t seed, uint64_t i) {
  uint64_t z = seed + (i + 1) * kGamma;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// floor(x * n / 2^64): maps a uniform 64-bit word onto [0, n).
WETRIC_HD uint64_t mulhi64(uint64_t x, uint64_t n) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(x, n);
#else
  return (uint64_t)(((unsigned __int128)x * n) >> 64);
#endif
}

// R-MAT quadrant thresholds as 32-bit fixed point (a, a+b, a+b+c).
struct RmatThresholds {
  uint32_t ta, tab, tabc;
};

inline RmatThresholds rmat_thresholds(double a, double b, double c) {
  auto fx = [](double p) -> uint32_t {
    double v = p * 4294967296.0;
    if (v <= 0.0) return 0u;
    if (v >= 4294967295.0) return 0xFFFFFFFFu;
    return (uint32_t)v;
  };
  RmatThresholds t;
  t.ta = fx(a);
  t.tab = fx(a + b);
  t.tabc = fx(a + b + c);
  return t;
}

// Edge k of a recursive-matrix (R-MAT, Chakrabarti et al. 2004) stream of
// scale `scale`: `scale` quadrant choices, most significant bit first;
// quadrant a = (0,0), b = (0,1), c = (1,0), d = (1,1). Two 32-bit uniforms
// are cut from each 64-bit draw.
WETRIC_HD void rmat_edge(uint64_t seed, uint32_t scale, RmatThresholds t,
                         uint64_t k, uint32_t *src, uint32_t *dst) {
  const uint64_t per_edge = (scale + 1) >> 1;
  uint32_t s = 0, d = 0;
  uint64_t r = 0;
  for (uint32_t l = 0; l < scale; ++l) {
    if ((l & 1u) == 0) r = splitmix64_at(seed, k * per_edge + (l >> 1));
    const uint32_t x = (l & 1u) ? (uint32_t)(r >> 32) : (uint32_t)r;
    const uint32_t bs = x >= t.tab ? 1u : 0u;
    const uint32_t bd = (x >= t.ta && x < t.tab) || x >= t.tabc ? 1u : 0u;
    s = (s << 1) | bs;
    d = (d << 1) | bd;
  }
  *src = s;
  *dst = d;
}

// Index of the first cdf entry > x (cdf non-decreasing, length n).
WETRIC_HD uint32_t cdf_upper_bound(const uint64_t *cdf, uint32_t n,
                                   uint64_t x) {
  uint32_t lo = 0, len = n;
  while (len > 0) {
    const uint32_t h = len >> 1;
    if (cdf[lo + h] <= x) {
      lo += h + 1;
      len -= h + 1;
    } else {
      len = h;
    }
  }
  return lo;
}

// Edge k of a weighted endpoint stream: each endpoint drawn independently
// with probability proportional to its integer weight (cdf = inclusive
// prefix of weights, total = cdf[n-1]). With power-law weights this is the
// Chung-Lu model sampled edge by edge (expected degree proportional to
// weight); with cdf == nullptr both endpoints are uniform on [0, n)
// (Erdos-Renyi G(n, M) with replacement).
WETRIC_HD void weighted_edge(uint64_t seed, const uint64_t *cdf, uint32_t n,
                             uint64_t k, uint32_t *src, uint32_t *dst) {
  const uint64_t r0 = splitmix64_at(seed, 2 * k);
  const uint64_t r1 = splitmix64_at(seed, 2 * k + 1);
  if (cdf == nullptr) {
    *src = (uint32_t)mulhi64(r0, n);
    *dst = (uint32_t)mulhi64(r1, n);
  } else {
    const uint64_t total = cdf[n - 1];
    *src = cdf_upper_bound(cdf, n, mulhi64(r0, total));
    *dst = cdf_upper_bound(cdf, n, mulhi64(r1, total));
  }
}

}  // namespace gen
}  // namespace wetric
