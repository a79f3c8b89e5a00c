/*
 * wetric_tools.h -- synthetic-input tools of libwetric: seeded graph
 * generators (host and device, identical streams) and a Matrix Market
 * writer. The reference has no counterpart (it only reads files,
 * tc.cu:561); these make the seeded graphs that stand in for its datasets.
 */
#ifndef WETRIC_TOOLS_H
#define WETRIC_TOOLS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* R-MAT stream on the host (OpenMP): edge k -> (src[k], dst[k]). */
int wetric_gen_rmat(uint32_t scale, uint64_t num_edges, double a, double b,
                    double c, uint64_t seed, uint32_t *src, uint32_t *dst);

/* Inclusive prefix of power-law integer weights for a Chung-Lu graph:
 * weight(i) = max(1, floor(2^32 * (1 + i / i0)^(-1 / (gamma - 1)))). */
int wetric_chung_lu_cdf(uint32_t n, double gamma, double i0, uint64_t *cdf);

/* Weighted endpoint stream on the host: both endpoints drawn from cdf
 * (Chung-Lu); cdf == NULL draws them uniformly on [0, n) (Erdos-Renyi). */
int wetric_gen_weighted(const uint64_t *cdf, uint32_t n, uint64_t num_edges,
                        uint64_t seed, uint32_t *src, uint32_t *dst);

/* The same streams written straight into device buffers. cdf is a device
 * pointer (or NULL for Erdos-Renyi). */
int wetric_gen_rmat_device(uint32_t scale, uint64_t num_edges, double a,
                           double b, double c, uint64_t seed, uint32_t *src,
                           uint32_t *dst, int device);
int wetric_gen_weighted_device(const uint64_t *cdf, uint32_t n,
                               uint64_t num_edges, uint64_t seed,
                               uint32_t *src, uint32_t *dst, int device);

/* Writes pairs as a "coordinate pattern symmetric" Matrix Market file,
 * 1-based, one "max min" line per pair (self-loops and repeats kept, so
 * the reader's cleanup is exercised). */
int wetric_write_mm(const char *path, uint64_t n, const uint32_t *src,
                    const uint32_t *dst, uint64_t num_pairs);

/* Host-only parse of a text edge list / Matrix Market file with the rules
 * of wetric_read_graph: *src / *dst receive malloc'd 0-based non-loop pairs
 * (release with wetric_free_buffer), *n = max id + 1. */
int wetric_parse_file(const char *path, int matrix_market, int zero_indexed,
                      uint32_t **src, uint32_t **dst, uint64_t *count,
                      uint64_t *n);
void wetric_free_buffer(void *p);

#ifdef __cplusplus
}
#endif

#endif /* WETRIC_TOOLS_H */
