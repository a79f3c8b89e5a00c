/*
 * oracle.c -- CPU oracle for the wedge-parallel triangle count.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product (the libwetric library,
 * the tc tool) links, loads or calls this file; only tests/, the smoke()
 * check of __graft_entry__.py and the cpu_baseline / reference legs of
 * bench.py use it, as the checker.
 *
 * It restates, in plain C, the reference's host pipeline and its count:
 *   oracle_read_graph     read_graph        tc.cu:561-685 (PREPROCESS_CPU
 *                         branch: qsort of the symmetrised edge list)
 *   oracle_csr_from_pairs the same from in-memory pairs
 *   oracle_preprocess     preprocess        tc.cu:687-787, with the vertex
 *                         order of the reference's default GPU styles (CUB's
 *                         stable radix sort by degree, tc.cu:494-498, 520-538):
 *                         ascending degree, ties by ascending id
 *   oracle_count_wedges   tc_GPU_kernel     tc.cu:173-293 + the bitmap and
 *                         prefix of tc_GPU  tc.cu:329-361: every wedge
 *                         (v; w < u in N+(v)) checked for edge (w, u), via the
 *                         bitmap for w in the last a vertices, else a linear
 *                         (d+ < 2) or binary search in N+(w)
 *   oracle_decode_wedge   the first-wedge decode of tc.cu:206-212 (double sqrt)
 *   oracle_count_merge    an independent count: sum over oriented edges (v, w)
 *                         of |N+(v) & N+(w)| by sorted merge (OpenMP)
 *   oracle_gen_rmat       the seeded R-MAT pair stream of the benchmark
 *   oracle_write_mm       pairs -> symmetric pattern Matrix Market file
 *                         (these two let the benchmark's reference arm make
 *                         its input file without loading the product library;
 *                         a CPU test checks the stream against the product's)
 * The two counts are independent algorithms; both count every triangle once
 * at its lowest-ranked vertex.
 *
 * Offsets are u64 throughout (the big-graph layout of
 * experiments/tc_big_graphs.cu:58-63), so one oracle covers both files.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  uint64_t n;
  uint64_t m;
  uint64_t *rp; /* n + 1 */
  uint32_t *ci; /* m */
} ocsr;

typedef struct {
  uint32_t src, dst;
} oedge;

void oracle_free(ocsr *g) {
  if (!g) return;
  free(g->rp);
  free(g->ci);
  g->rp = NULL;
  g->ci = NULL;
  g->n = g->m = 0;
}

/* compareEdge_t, tc.cu:470-478 */
static int cmp_edge(const void *a, const void *b) {
  const oedge *x = (const oedge *)a, *y = (const oedge *)b;
  if (x->src != y->src) return x->src < y->src ? -1 : 1;
  if (x->dst != y->dst) return x->dst < y->dst ? -1 : 1;
  return 0;
}

static int cmp_u32(const void *a, const void *b) {
  const uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}

/* Sort + dedup + CSR of a symmetrised directed edge list (tc.cu:646-684).
 * Takes ownership of `edges`. */
static int csr_from_directed(oedge *edges, uint64_t count, uint64_t n,
                             ocsr *out) {
  memset(out, 0, sizeof(*out));
  out->n = n;
  out->rp = (uint64_t *)calloc(n + 1, sizeof(uint64_t));
  if (!out->rp) {
    free(edges);
    return -1;
  }
  if (count == 0) {
    /* The reference reads edges[0] uninitialised here; an empty graph is
     * the defined answer. */
    out->ci = (uint32_t *)malloc(sizeof(uint32_t));
    free(edges);
    return out->ci ? 0 : -1;
  }
  qsort(edges, count, sizeof(oedge), cmp_edge);
  uint32_t *ci = (uint32_t *)malloc(count * sizeof(uint32_t));
  if (!ci) {
    free(edges);
    return -1;
  }
  uint64_t k = 0;
  for (uint64_t i = 0; i < count; ++i) {
    if (i == 0 || cmp_edge(&edges[i - 1], &edges[i]) != 0) {
      ci[k++] = edges[i].dst;
      out->rp[edges[i].src + 1]++;
    }
  }
  for (uint64_t v = 1; v <= n; ++v) out->rp[v] += out->rp[v - 1];
  free(edges);
  out->m = k;
  out->ci = ci;
  return 0;
}

/* read_graph, tc.cu:561-685. Returns 0, or -1 (cannot open / allocate),
 * -2 (no data line: the reference's usage() exit), -3 (zero id without
 * zero_indexed: tc.cu:599-602). */
int oracle_read_graph(const char *path, int matrix_market, int zero_indexed,
                      ocsr *out) {
  FILE *f = fopen(path, "r");
  if (!f) return -1;
  char line[256];
  do {
    if (fgets(line, sizeof(line), f) == NULL) {
      fclose(f);
      return -2;
    }
  } while (line[0] < '0' || line[0] > '9');
  if (matrix_market) {
    if (fgets(line, sizeof(line), f) == NULL) {
      fclose(f);
      return -2;
    }
  }
  uint64_t cap = 10240, count = 0;
  oedge *edges = (oedge *)malloc(cap * sizeof(oedge));
  if (!edges) {
    fclose(f);
    return -1;
  }
  uint32_t max_vertex = 0;
  unsigned int v, w;
  if (sscanf(line, "%u %u\n", &v, &w) == 2) {
    do {
      if (count + 2 > cap) {
        cap *= 2;
        oedge *ne = (oedge *)realloc(edges, cap * sizeof(oedge));
        if (!ne) {
          free(edges);
          fclose(f);
          return -1;
        }
        edges = ne;
      }
      if (!zero_indexed && (v == 0 || w == 0)) {
        free(edges);
        fclose(f);
        return -3;
      }
      if (!zero_indexed) {
        v -= 1;
        w -= 1;
      }
      if (v != w) {
        if (v > max_vertex) max_vertex = v;
        if (w > max_vertex) max_vertex = w;
        edges[count].src = v;
        edges[count].dst = w;
        count++;
        edges[count].src = w;
        edges[count].dst = v;
        count++;
      }
    } while (fscanf(f, "%u %u\n", &v, &w) == 2);
  }
  fclose(f);
  return csr_from_directed(edges, count, (uint64_t)max_vertex + 1, out) ? -1
                                                                        : 0;
}

/* read_graph on in-memory 0-based pairs (self-loops dropped, both
 * directions kept, n = max id + 1 over non-loop pairs, or n_hint). */
int oracle_csr_from_pairs(const uint32_t *src, const uint32_t *dst,
                          uint64_t count, uint64_t n_hint, ocsr *out) {
  oedge *edges = (oedge *)malloc((2 * count + 1) * sizeof(oedge));
  if (!edges) return -1;
  uint64_t k = 0;
  uint32_t max_vertex = 0;
  for (uint64_t i = 0; i < count; ++i) {
    const uint32_t v = src[i], w = dst[i];
    if (v == w) continue;
    if (v > max_vertex) max_vertex = v;
    if (w > max_vertex) max_vertex = w;
    edges[k].src = v;
    edges[k].dst = w;
    k++;
    edges[k].src = w;
    edges[k].dst = v;
    k++;
  }
  const uint64_t n = n_hint ? n_hint : (uint64_t)max_vertex + 1;
  return csr_from_directed(edges, k, n, out);
}

typedef struct {
  uint32_t id;
  uint64_t deg;
} overtex;

static int cmp_vertex(const void *a, const void *b) {
  const overtex *x = (const overtex *)a, *y = (const overtex *)b;
  if (x->deg != y->deg) return x->deg < y->deg ? -1 : 1;
  return x->id < y->id ? -1 : (x->id > y->id ? 1 : 0);
}

/* preprocess, tc.cu:687-787 (stable degree order). */
int oracle_preprocess(const ocsr *in, ocsr *out) {
  const uint64_t n = in->n;
  memset(out, 0, sizeof(*out));
  overtex *vs = (overtex *)malloc((n ? n : 1) * sizeof(overtex));
  uint32_t *rev = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
  if (!vs || !rev) {
    free(vs);
    free(rev);
    return -1;
  }
  for (uint64_t v = 0; v < n; ++v) {
    vs[v].id = (uint32_t)v;
    vs[v].deg = in->rp[v + 1] - in->rp[v];
  }
  qsort(vs, n, sizeof(overtex), cmp_vertex);
  for (uint64_t v = 0; v < n; ++v) rev[vs[v].id] = (uint32_t)v;
  out->n = n;
  out->rp = (uint64_t *)malloc((n + 1) * sizeof(uint64_t));
  out->ci = (uint32_t *)malloc((in->m ? in->m : 1) * sizeof(uint32_t));
  if (!out->rp || !out->ci) {
    free(vs);
    free(rev);
    oracle_free(out);
    return -1;
  }
  uint64_t k = 0;
  out->rp[0] = 0;
  for (uint64_t v = 0; v < n; ++v) {
    const uint32_t old = vs[v].id;
    const uint64_t start = k;
    for (uint64_t j = in->rp[old]; j < in->rp[old + 1]; ++j) {
      const uint32_t wn = rev[in->ci[j]];
      if (wn > v) out->ci[k++] = wn;
    }
    qsort(out->ci + start, k - start, sizeof(uint32_t), cmp_u32);
    out->rp[v + 1] = k;
  }
  out->m = k;
  free(vs);
  free(rev);
  return 0;
}

/* W = sum over v of C(d+(v), 2) (tc.cu:348-361, in u64). */
uint64_t oracle_wedge_total(const ocsr *g) {
  uint64_t W = 0;
  for (uint64_t v = 0; v < g->n; ++v) {
    const uint64_t d = g->rp[v + 1] - g->rp[v];
    if (d >= 2) W += d * (d - 1) / 2;
  }
  return W;
}

/* Out-degree bound of the oriented CSR. */
uint64_t oracle_max_out_degree(const ocsr *g) {
  uint64_t mx = 0;
  for (uint64_t v = 0; v < g->n; ++v) {
    const uint64_t d = g->rp[v + 1] - g->rp[v];
    if (d > mx) mx = d;
  }
  return mx;
}

/* The reference's first-wedge decode (tc.cu:206-212, the u64 form of
 * experiments/tc_big_graphs.cu:206-212). */
void oracle_decode_wedge(uint64_t iv, uint64_t d, uint64_t *wi, uint64_t *ui) {
  const uint64_t wedges = d * (d - 1) / 2;
  const uint64_t w_i =
      d - 2 - (uint64_t)(sqrt(((double)(wedges - iv) - 0.875) * 2) - 0.5);
  *wi = w_i;
  *ui = iv + w_i + 1 + (((d - w_i) * (d - w_i - 1)) / 2 - wedges);
}

/* binary_search_GPU / linear_search_GPU, tc.cu:89-114: is u in
 * ci[b, e)? */
static int edge_exists(const uint32_t *ci, uint64_t b, uint64_t e, uint32_t u) {
  if (e - b < 2) {
    for (uint64_t i = b; i < e; ++i) {
      if (ci[i] == u) return 1;
      if (ci[i] > u) break;
    }
    return 0;
  }
  uint64_t s = b, t = e;
  while (s < t) {
    const uint64_t mid = (s + t) >> 1;
    if (ci[mid] == u) return 1;
    if (ci[mid] < u) s = mid + 1;
    else t = mid;
  }
  return 0;
}

/* Wedge-check count of wedges [wb, we) (we == 0: to W) with bitmap length
 * a (tc.cu:173-293 with the host-built bitmap of tc.cu:329-346). Wedge order:
 * v ascending, then (w_i, u_i) row-major. */
uint64_t oracle_count_wedges(const ocsr *g, uint64_t wb, uint64_t we,
                             uint32_t a) {
  const uint64_t n = g->n;
  const uint64_t W = oracle_wedge_total(g);
  if (we == 0 || we > W) we = W;
  if (wb >= we) return 0;
  /* Bitmap over the last a vertices; ceiling word count. */
  const uint64_t S = (uint64_t)a * (a ? a - 1 : 0) / 2;
  const uint64_t first = (n > a ? n : a) - a;
  uint32_t *bm = (uint32_t *)calloc((S + 31) / 32 + 1, sizeof(uint32_t));
  if (!bm) return UINT64_MAX;
  for (uint64_t v = n - (n < a ? n : a); v < n; ++v)
    for (uint64_t j = g->rp[v]; j < g->rp[v + 1]; ++j) {
      const uint64_t w = g->ci[j];
      const uint64_t idx = S - (n - v) * (n - v - 1) / 2 + w - v - 1;
      bm[idx >> 5] |= 1u << (idx & 31);
    }
  /* wedge prefix */
  uint64_t *ws = (uint64_t *)malloc((n + 1) * sizeof(uint64_t));
  if (!ws) {
    free(bm);
    return UINT64_MAX;
  }
  ws[0] = 0;
  for (uint64_t v = 0; v < n; ++v) {
    const uint64_t d = g->rp[v + 1] - g->rp[v];
    ws[v + 1] = ws[v] + (d >= 2 ? d * (d - 1) / 2 : 0);
  }
  uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
  for (int64_t vv = 0; vv < (int64_t)n; ++vv) {
    const uint64_t v = (uint64_t)vv;
    if (ws[v + 1] <= wb || ws[v] >= we) continue;
    const uint64_t rb = g->rp[v], d = g->rp[v + 1] - rb;
    uint64_t i = ws[v];
    for (uint64_t wi = 0; wi + 1 < d; ++wi) {
      const uint64_t row_end = i + (d - wi - 1);
      if (row_end <= wb || i >= we) {
        i = row_end;
        continue;
      }
      const uint32_t w = g->ci[rb + wi];
      for (uint64_t ui = wi + 1; ui < d; ++ui, ++i) {
        if (i < wb || i >= we) continue;
        const uint32_t u = g->ci[rb + ui];
        int hit;
        if ((uint64_t)w >= first) {
          const uint64_t idx = S - (n - w) * (n - w - 1) / 2 + u - w - 1;
          hit = (bm[idx >> 5] >> (idx & 31)) & 1u;
        } else {
          hit = edge_exists(g->ci, g->rp[w], g->rp[w + 1], u);
        }
        total += (uint64_t)hit;
      }
    }
  }
  free(ws);
  free(bm);
  return total;
}

/* |N+(v) & N+(w)| summed over oriented edges (v, w) with v in
 * [vbegin, vend) (vend == 0: n). OpenMP over v. */
uint64_t oracle_count_merge_range(const ocsr *g, uint64_t vbegin,
                                  uint64_t vend) {
  if (vend == 0 || vend > g->n) vend = g->n;
  uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total)
  for (int64_t vv = (int64_t)vbegin; vv < (int64_t)vend; ++vv) {
    const uint64_t v = (uint64_t)vv;
    const uint64_t vb = g->rp[v], ve = g->rp[v + 1];
    for (uint64_t j = vb; j < ve; ++j) {
      const uint32_t w = g->ci[j];
      uint64_t p = j + 1, q = g->rp[w];
      const uint64_t qe = g->rp[w + 1];
      while (p < ve && q < qe) {
        const uint32_t x = g->ci[p], y = g->ci[q];
        if (x == y) {
          ++total;
          ++p;
          ++q;
        } else if (x < y) {
          ++p;
        } else {
          ++q;
        }
      }
    }
  }
  return total;
}

uint64_t oracle_count_merge(const ocsr *g) {
  return oracle_count_merge_range(g, 0, 0);
}

/* Wedges of the vertices [vbegin, vend). */
uint64_t oracle_wedges_range(const ocsr *g, uint64_t vbegin, uint64_t vend) {
  if (vend == 0 || vend > g->n) vend = g->n;
  uint64_t W = 0;
  for (uint64_t v = vbegin; v < vend; ++v) {
    const uint64_t d = g->rp[v + 1] - g->rp[v];
    if (d >= 2) W += d * (d - 1) / 2;
  }
  return W;
}

/* Algorithmic bytes of the wedge-check count: 8(n+1) + 4m + 8(n+1) streamed
 * once, plus 4 + 16 + 4*ceil(log2(d+(w) + 1)) per wedge with middle w. */
uint64_t oracle_algorithmic_bytes(const ocsr *g) {
  uint64_t B = 8 * (g->n + 1) + 4 * g->m + 8 * (g->n + 1);
  for (uint64_t v = 0; v < g->n; ++v) {
    const uint64_t b = g->rp[v], e = g->rp[v + 1];
    for (uint64_t j = b; j < e; ++j) {
      const uint64_t wedges = e - j - 1;
      if (!wedges) continue;
      const uint32_t w = g->ci[j];
      const uint64_t dw = g->rp[w + 1] - g->rp[w];
      uint64_t bits = 0;
      while ((dw >> bits) != 0) ++bits;
      B += wedges * (4 + 16 + 4 * bits);
    }
  }
  return B;
}

int oracle_max_threads(void) { return omp_get_max_threads(); }

/* ------------------------------------------------------------------------
 * Seeded R-MAT pairs (Chakrabarti, Zhan, Faloutsos, "R-MAT: A Recursive
 * Model for Graph Mining", SDM 2004): `scale` quadrant choices per edge,
 * most significant bit first, quadrant a = (0,0), b = (0,1), c = (1,0),
 * d = (1,1). The uniforms are the splitmix64 output function (Steele, Lea,
 * Flood, OOPSLA 2014) at seed + (i + 1) * golden gamma, two 32-bit uniforms
 * per 64-bit draw, compared with 32-bit fixed-point thresholds, so the
 * stream is a pure function of (seed, edge index).
 * ---------------------------------------------------------------------- */
static uint64_t sm64_at(uint64_t seed, uint64_t i) {
  uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static uint32_t fixed32(double p) {
  const double v = p * 4294967296.0;
  if (v <= 0.0) return 0u;
  if (v >= 4294967295.0) return 0xFFFFFFFFu;
  return (uint32_t)v;
}

int oracle_gen_rmat(uint32_t scale, uint64_t count, double a, double b,
                    double c, uint64_t seed, uint32_t *src, uint32_t *dst) {
  if (scale == 0 || scale > 32) return -1;
  const uint32_t ta = fixed32(a), tab = fixed32(a + b), tabc = fixed32(a + b + c);
  const uint64_t per_edge = (scale + 1) >> 1;
#pragma omp parallel for schedule(static)
  for (int64_t kk = 0; kk < (int64_t)count; ++kk) {
    const uint64_t k = (uint64_t)kk;
    uint32_t sv = 0, dv = 0;
    uint64_t r = 0;
    for (uint32_t l = 0; l < scale; ++l) {
      if ((l & 1u) == 0) r = sm64_at(seed, k * per_edge + (l >> 1));
      const uint32_t x = (l & 1u) ? (uint32_t)(r >> 32) : (uint32_t)r;
      sv = (sv << 1) | (x >= tab ? 1u : 0u);
      dv = (dv << 1) | (((x >= ta && x < tab) || x >= tabc) ? 1u : 0u);
    }
    src[k] = sv;
    dst[k] = dv;
  }
  return 0;
}

/* Pairs as "coordinate pattern symmetric" Matrix Market: a banner, the size
 * line "n n count", then one 1-based "max min" line per pair (the input form
 * the reference's read_graph takes with -m, tc.cu:561-621). */
int oracle_write_mm(const char *path, uint64_t n, const uint32_t *src,
                    const uint32_t *dst, uint64_t count) {
  FILE *f = fopen(path, "wb");
  if (!f) return -1;
  static char buf[1 << 20];
  setvbuf(f, buf, _IOFBF, sizeof(buf));
  int ok = fprintf(f, "%%%%MatrixMarket matrix coordinate pattern symmetric\n"
                      "%llu %llu %llu\n",
                   (unsigned long long)n, (unsigned long long)n,
                   (unsigned long long)count) > 0;
  for (uint64_t i = 0; i < count && ok; ++i) {
    const uint32_t s = src[i], d = dst[i];
    ok = fprintf(f, "%llu %llu\n", (unsigned long long)(s > d ? s : d) + 1,
                 (unsigned long long)(s > d ? d : s) + 1) > 0;
  }
  if (fclose(f) != 0) ok = 0;
  return ok ? 0 : -1;
}

/* W and the max out-degree of the oriented graph of raw pairs, without
 * building the CSR (the same rules as oracle_csr_from_pairs +
 * oracle_preprocess): unique undirected edges, self-loops dropped, vertex
 * rank = stable (degree, id) order, each edge charged to its lower-ranked
 * end. Canonical (min, max) keys are sorted by an LSD radix sort (16-bit
 * digits), the ranks by a stable counting sort on the degree. */
int oracle_wedge_total_from_pairs(const uint32_t *src, const uint32_t *dst,
                                  uint64_t count, uint64_t *W_out,
                                  uint64_t *maxdeg_out) {
  uint64_t *k = (uint64_t *)malloc((count ? count : 1) * sizeof(uint64_t));
  uint64_t *t = (uint64_t *)malloc((count ? count : 1) * sizeof(uint64_t));
  if (!k || !t) {
    free(k);
    free(t);
    return -1;
  }
  uint64_t c = 0;
  uint32_t maxv = 0;
  for (uint64_t i = 0; i < count; ++i) {
    const uint32_t a = src[i], b = dst[i];
    if (a == b) continue;
    const uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
    if (hi > maxv) maxv = hi;
    k[c++] = ((uint64_t)lo << 32) | hi;
  }
  static uint64_t hist[65536];
  for (int pass = 0; pass < 4; ++pass) {
    const int sh = 16 * pass;
    memset(hist, 0, sizeof(hist));
    for (uint64_t i = 0; i < c; ++i) hist[(k[i] >> sh) & 0xFFFF]++;
    uint64_t run = 0;
    for (int d = 0; d < 65536; ++d) {
      const uint64_t h = hist[d];
      hist[d] = run;
      run += h;
    }
    for (uint64_t i = 0; i < c; ++i) t[hist[(k[i] >> sh) & 0xFFFF]++] = k[i];
    uint64_t *x = k;
    k = t;
    t = x;
  }
  const uint64_t n = c ? (uint64_t)maxv + 1 : 1;
  uint64_t *deg = (uint64_t *)calloc(n, sizeof(uint64_t));
  uint32_t *rank = (uint32_t *)malloc(n * sizeof(uint32_t));
  uint64_t *dplus = (uint64_t *)calloc(n, sizeof(uint64_t));
  if (!deg || !rank || !dplus) {
    free(k); free(t); free(deg); free(rank); free(dplus);
    return -1;
  }
  uint64_t u = 0;
  for (uint64_t i = 0; i < c; ++i) {
    if (i > 0 && k[i] == k[i - 1]) continue;
    k[u++] = k[i];
    deg[k[i] >> 32]++;
    deg[k[i] & 0xFFFFFFFFu]++;
  }
  uint64_t maxd = 0;
  for (uint64_t v = 0; v < n; ++v) maxd = deg[v] > maxd ? deg[v] : maxd;
  /* stable counting sort by degree: rank[v] = position of v */
  uint64_t *start = (uint64_t *)calloc(maxd + 2, sizeof(uint64_t));
  if (!start) {
    free(k); free(t); free(deg); free(rank); free(dplus);
    return -1;
  }
  for (uint64_t v = 0; v < n; ++v) start[deg[v] + 1]++;
  for (uint64_t d = 1; d <= maxd + 1; ++d) start[d] += start[d - 1];
  for (uint64_t v = 0; v < n; ++v) rank[v] = (uint32_t)start[deg[v]]++;
  for (uint64_t i = 0; i < u; ++i) {
    const uint32_t a = (uint32_t)(k[i] >> 32), b = (uint32_t)k[i];
    dplus[rank[a] < rank[b] ? a : b]++;
  }
  uint64_t W = 0, md = 0;
  for (uint64_t v = 0; v < n; ++v) {
    const uint64_t d = dplus[v];
    if (d >= 2) W += d * (d - 1) / 2;
    if (d > md) md = d;
  }
  *W_out = W;
  *maxdeg_out = md;
  free(k); free(t); free(deg); free(rank); free(dplus); free(start);
  return 0;
}
