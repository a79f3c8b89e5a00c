// tools.cu -- seeded generators (host loops and device kernels over the
// same per-edge functions of gen.cuh) and a parallel Matrix Market writer.
#include <cuda_runtime.h>
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <vector>

#include "common.cuh"
#include "gen.cuh"
#include "wetric_tools.h"

using namespace wetric;

namespace {

__global__ void k_gen_rmat(uint32_t scale, uint64_t E, gen::RmatThresholds t,
                           uint64_t seed, uint32_t *__restrict__ src,
                           uint32_t *__restrict__ dst) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < E;
       k += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t s, d;
    gen::rmat_edge(seed, scale, t, k, &s, &d);
    src[k] = s;
    dst[k] = d;
  }
}

__global__ void k_gen_weighted(const uint64_t *__restrict__ cdf, uint32_t n,
                               uint64_t E, uint64_t seed,
                               uint32_t *__restrict__ src,
                               uint32_t *__restrict__ dst) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < E;
       k += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t s, d;
    gen::weighted_edge(seed, cdf, n, k, &s, &d);
    src[k] = s;
    dst[k] = d;
  }
}

int finish_tool(int st) {
  if (st == WETRIC_OK) clear_error();
  return st;
}

// Appends the decimal form of x.
inline char *put_u64(char *p, uint64_t x) {
  char tmp[24];
  int k = 0;
  do {
    tmp[k++] = (char)('0' + x % 10);
    x /= 10;
  } while (x);
  while (k) *p++ = tmp[--k];
  return p;
}

}  // namespace

extern "C" {

int wetric_gen_rmat(uint32_t scale, uint64_t E, double a, double b, double c,
                    uint64_t seed, uint32_t *src, uint32_t *dst) {
  if (scale == 0 || scale > 32 || (E && (!src || !dst))) {
    set_error(WETRIC_EINVAL, "bad R-MAT arguments");
    return WETRIC_EINVAL;
  }
  const gen::RmatThresholds t = gen::rmat_thresholds(a, b, c);
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < (int64_t)E; ++k)
    gen::rmat_edge(seed, scale, t, (uint64_t)k, src + k, dst + k);
  return finish_tool(WETRIC_OK);
}

int wetric_chung_lu_cdf(uint32_t n, double gamma, double i0, uint64_t *cdf) {
  if (n == 0 || !cdf || gamma <= 1.0 || i0 <= 0.0) {
    set_error(WETRIC_EINVAL, "bad Chung-Lu arguments");
    return WETRIC_EINVAL;
  }
  const double alpha = 1.0 / (gamma - 1.0);
  std::vector<uint64_t> w(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    double x = 4294967296.0 * pow(1.0 + (double)i / i0, -alpha);
    uint64_t q = (uint64_t)x;
    w[i] = q ? q : 1;
  }
  uint64_t run = 0;
  for (uint32_t i = 0; i < n; ++i) {
    run += w[i];
    cdf[i] = run;
  }
  return finish_tool(WETRIC_OK);
}

int wetric_gen_weighted(const uint64_t *cdf, uint32_t n, uint64_t E,
                        uint64_t seed, uint32_t *src, uint32_t *dst) {
  if (n == 0 || (E && (!src || !dst))) {
    set_error(WETRIC_EINVAL, "bad generator arguments");
    return WETRIC_EINVAL;
  }
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < (int64_t)E; ++k)
    gen::weighted_edge(seed, cdf, n, (uint64_t)k, src + k, dst + k);
  return finish_tool(WETRIC_OK);
}

int wetric_gen_rmat_device(uint32_t scale, uint64_t E, double a, double b,
                           double c, uint64_t seed, uint32_t *src,
                           uint32_t *dst, int device) {
  if (scale == 0 || scale > 32 || (E && (!src || !dst))) {
    set_error(WETRIC_EINVAL, "bad R-MAT arguments");
    return WETRIC_EINVAL;
  }
  DeviceContext *ctx = nullptr;
  int st = get_context(device, &ctx);
  if (st != WETRIC_OK) return st;
  auto run = [&]() -> int {
    if (E) {
      uint64_t g = ceil_div(E, 256);
      const uint64_t cap = (uint64_t)ctx->sm_count * 16;
      if (g > cap) g = cap;
      k_gen_rmat<<<(unsigned)g, 256, 0, ctx->stream>>>(
          scale, E, gen::rmat_thresholds(a, b, c), seed, src, dst);
      WETRIC_LAUNCH_CHECK();
    }
    WETRIC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return WETRIC_OK;
  };
  return finish_tool(run());
}

int wetric_gen_weighted_device(const uint64_t *cdf, uint32_t n, uint64_t E,
                               uint64_t seed, uint32_t *src, uint32_t *dst,
                               int device) {
  if (n == 0 || (E && (!src || !dst))) {
    set_error(WETRIC_EINVAL, "bad generator arguments");
    return WETRIC_EINVAL;
  }
  DeviceContext *ctx = nullptr;
  int st = get_context(device, &ctx);
  if (st != WETRIC_OK) return st;
  auto run = [&]() -> int {
    if (E) {
      uint64_t g = ceil_div(E, 256);
      const uint64_t cap = (uint64_t)ctx->sm_count * 16;
      if (g > cap) g = cap;
      k_gen_weighted<<<(unsigned)g, 256, 0, ctx->stream>>>(cdf, n, E, seed,
                                                           src, dst);
      WETRIC_LAUNCH_CHECK();
    }
    WETRIC_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return WETRIC_OK;
  };
  return finish_tool(run());
}

int wetric_write_mm(const char *path, uint64_t n, const uint32_t *src,
                    const uint32_t *dst, uint64_t P) {
  if (!path || (P && (!src || !dst))) {
    set_error(WETRIC_EINVAL, "bad writer arguments");
    return WETRIC_EINVAL;
  }
  FILE *f = fopen(path, "wb");
  if (!f) {
    set_error(WETRIC_EIO, "cannot open %s for writing", path);
    return WETRIC_EIO;
  }
  fprintf(f, "%%%%MatrixMarket matrix coordinate pattern symmetric\n");
  fprintf(f, "%llu %llu %llu\n", (unsigned long long)n, (unsigned long long)n,
          (unsigned long long)P);
  const uint64_t chunk = 1ull << 20;
  const uint64_t nchunks = (P + chunk - 1) / chunk;
  const int threads = omp_get_max_threads();
  std::vector<std::vector<char>> bufs(threads);
  bool ok = true;
  for (uint64_t c0 = 0; c0 < nchunks && ok; c0 += (uint64_t)threads) {
    const uint64_t c1 = c0 + threads < nchunks ? c0 + threads : nchunks;
#pragma omp parallel for schedule(static, 1) num_threads(threads)
    for (int64_t c = (int64_t)c0; c < (int64_t)c1; ++c) {
      std::vector<char> &b = bufs[c - c0];
      const uint64_t lo = (uint64_t)c * chunk;
      const uint64_t hi = lo + chunk < P ? lo + chunk : P;
      b.resize((hi - lo) * 24);
      char *p = b.data();
      for (uint64_t i = lo; i < hi; ++i) {
        const uint32_t s = src[i], d = dst[i];
        p = put_u64(p, (uint64_t)(s > d ? s : d) + 1);
        *p++ = ' ';
        p = put_u64(p, (uint64_t)(s > d ? d : s) + 1);
        *p++ = '\n';
      }
      b.resize((size_t)(p - b.data()));
    }
    for (uint64_t c = c0; c < c1 && ok; ++c) {
      std::vector<char> &b = bufs[c - c0];
      if (!b.empty() && fwrite(b.data(), 1, b.size(), f) != b.size()) ok = false;
    }
  }
  if (fclose(f) != 0) ok = false;
  if (!ok) {
    set_error(WETRIC_EIO, "write to %s failed", path);
    return WETRIC_EIO;
  }
  return finish_tool(WETRIC_OK);
}

}  // extern "C"
