// graph_io.cpp -- parallel text edge-list / Matrix Market parser.
//
// Follows the input rules of read_graph (tc.cu:561-625):
//   * leading lines whose first character is not a digit are skipped
//     (comments, the %%MatrixMarket banner, blank lines), tc.cu:572-574;
//   * for Matrix Market one more line (the size line) is skipped,
//     tc.cu:577-579 -- its counts are not used;
//   * every following line gives "v w"; ids are 1-based unless
//     zero_indexed, and a zero id without zero_indexed is an error
//     (tc.cu:599-602); self-loops are dropped (tc.cu:608);
//   * n = (largest id among non-loop pairs) + 1 (tc.cu:625).
// Deliberate differences, all on inputs the reference mis-reads:
//   * the reference reads the body as a token stream with fscanf("%d %d"),
//     so a third column shifts or ends the parse; here parsing is per line
//     and any further columns on a line are ignored;
//   * the reference stops silently at the first unparsable token; here the
//     parse also stops at the first line that does not start with two
//     integers (blank lines are skipped, like fscanf's whitespace skip);
//   * negative ids or ids >= 2^32 are rejected (the reference wraps them
//     through "%d" into an unsigned).
// The body is split into one chunk per thread at line boundaries.
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "graph_io.h"
#include "wetric_tools.h"

namespace wetric {

namespace {

inline bool is_digit(char c) { return c >= '0' && c <= '9'; }
inline bool is_space(char c) {
  return c == ' ' || c == '\t' || c == '\r' || c == '\f' || c == '\v';
}

// Parses one line [p, end) (no '\n'). Returns 1 with (v, w) set, 0 for a
// blank line, -1 for a line that does not start with two integers, -2 for
// an id outside [0, 2^32).
int parse_line(const char *p, const char *end, int64_t *v, int64_t *w) {
  while (p < end && is_space(*p)) ++p;
  if (p == end) return 0;
  int64_t vals[2];
  for (int k = 0; k < 2; ++k) {
    while (p < end && is_space(*p)) ++p;
    bool neg = false;
    if (p < end && (*p == '-' || *p == '+')) {
      neg = *p == '-';
      ++p;
    }
    if (p == end || !is_digit(*p)) return -1;
    uint64_t x = 0;
    while (p < end && is_digit(*p)) {
      x = x * 10 + (uint64_t)(*p - '0');
      if (x > 0xFFFFFFFFull) {
        // keep consuming digits; the value is out of range either way
        while (p < end && is_digit(*p)) ++p;
        return -2;
      }
      ++p;
    }
    if (neg && x != 0) return -2;
    // The first id must be followed by whitespace; anything after the
    // second id (a weight column, say) is ignored.
    if (k == 0 && p < end && !is_space(*p)) return -1;
    vals[k] = (int64_t)x;
  }
  *v = vals[0];
  *w = vals[1];
  return 1;
}

struct Chunk {
  std::vector<uint32_t> src, dst;
  uint32_t max_id = 0;
  bool any = false;
  bool stopped = false;  // hit a line that ends the parse
  int error = 0;         // WETRIC_EINVAL (zero id) or WETRIC_EIO
  uint64_t error_line_offset = 0;
};

}  // namespace

int parse_edge_text(const char *data, size_t size, bool matrix_market,
                    bool zero_indexed, std::vector<uint32_t> *src,
                    std::vector<uint32_t> *dst, uint64_t *n_out,
                    std::string *msg) {
  size_t pos = 0;
  // Header: skip lines whose first character is not a digit.
  for (;;) {
    if (pos >= size) {
      *msg = "no data line in graph file";
      return WETRIC_EIO;
    }
    const char *nl = (const char *)memchr(data + pos, '\n', size - pos);
    const size_t line_end = nl ? (size_t)(nl - data) : size;
    if (is_digit(data[pos])) break;
    pos = nl ? line_end + 1 : size;
  }
  if (matrix_market) {
    const char *nl = (const char *)memchr(data + pos, '\n', size - pos);
    if (!nl) {
      *msg = "Matrix Market file ends after its size line";
      return WETRIC_EIO;
    }
    pos = (size_t)(nl - data) + 1;
  }

  const size_t body = size - pos;
  int threads = omp_get_max_threads();
  if (body < (1u << 20)) threads = 1;
  std::vector<size_t> cut(threads + 1);
  cut[0] = pos;
  cut[threads] = size;
  for (int t = 1; t < threads; ++t) {
    size_t c = pos + body * (size_t)t / (size_t)threads;
    if (c < cut[t - 1]) c = cut[t - 1];
    const char *nl = (const char *)memchr(data + c, '\n', size - c);
    cut[t] = nl ? (size_t)(nl - data) + 1 : size;
  }
  std::vector<Chunk> chunks(threads);
#pragma omp parallel for schedule(static, 1) num_threads(threads)
  for (int t = 0; t < threads; ++t) {
    Chunk &ck = chunks[t];
    size_t p = cut[t];
    const size_t end = cut[t + 1];
    ck.src.reserve((end - p) / 8 + 16);
    ck.dst.reserve((end - p) / 8 + 16);
    while (p < end) {
      const char *nl = (const char *)memchr(data + p, '\n', end - p);
      const size_t le = nl ? (size_t)(nl - data) : end;
      int64_t v = 0, w = 0;
      const int r = parse_line(data + p, data + le, &v, &w);
      if (r < 0) {
        ck.stopped = true;
        if (r == -2) {
          ck.error = WETRIC_EIO;
          ck.error_line_offset = p;
        }
        break;
      }
      if (r == 1) {
        if (!zero_indexed && (v == 0 || w == 0)) {
          ck.stopped = true;
          ck.error = WETRIC_EINVAL;
          ck.error_line_offset = p;
          break;
        }
        if (!zero_indexed) {
          --v;
          --w;
        }
        if (v != w) {
          ck.src.push_back((uint32_t)v);
          ck.dst.push_back((uint32_t)w);
          const uint32_t mx = (uint32_t)(v > w ? v : w);
          if (mx > ck.max_id) ck.max_id = mx;
          ck.any = true;
        }
      }
      p = nl ? le + 1 : end;
    }
  }
  // Chunks after the first stopped one are not part of the parse.
  size_t total = 0;
  uint32_t max_id = 0;
  int last = threads - 1;
  for (int t = 0; t < threads; ++t) {
    if (chunks[t].error) {
      *msg = chunks[t].error == WETRIC_EINVAL
                 ? "zero vertex id detected but zero-indexing was not set"
                 : "vertex id outside [0, 2^32)";
      return chunks[t].error;
    }
    total += chunks[t].src.size();
    if (chunks[t].any && chunks[t].max_id > max_id) max_id = chunks[t].max_id;
    if (chunks[t].stopped) {
      last = t;
      break;
    }
  }
  src->resize(total);
  dst->resize(total);
  std::vector<size_t> off(last + 2, 0);
  for (int t = 0; t <= last; ++t) off[t + 1] = off[t] + chunks[t].src.size();
#pragma omp parallel for schedule(static, 1) num_threads(threads)
  for (int t = 0; t <= last; ++t) {
    if (!chunks[t].src.empty()) {
      memcpy(src->data() + off[t], chunks[t].src.data(),
             chunks[t].src.size() * sizeof(uint32_t));
      memcpy(dst->data() + off[t], chunks[t].dst.data(),
             chunks[t].dst.size() * sizeof(uint32_t));
    }
  }
  *n_out = (uint64_t)max_id + 1;
  return WETRIC_OK;
}

int parse_edge_file(const char *path, bool matrix_market, bool zero_indexed,
                    std::vector<uint32_t> *src, std::vector<uint32_t> *dst,
                    uint64_t *n_out, std::string *msg) {
  FILE *f = fopen(path, "rb");
  if (!f) {
    *msg = std::string("unable to open graph file ") + path;
    return WETRIC_EIO;
  }
  if (fseek(f, 0, SEEK_END) != 0) {
    fclose(f);
    *msg = "unable to seek graph file";
    return WETRIC_EIO;
  }
  const long sz = ftell(f);
  if (sz < 0) {
    fclose(f);
    *msg = "unable to size graph file";
    return WETRIC_EIO;
  }
  fseek(f, 0, SEEK_SET);
  std::vector<char> buf((size_t)sz + 1);
  const size_t got = sz ? fread(buf.data(), 1, (size_t)sz, f) : 0;
  fclose(f);
  if (got != (size_t)sz) {
    *msg = "short read on graph file";
    return WETRIC_EIO;
  }
  buf[(size_t)sz] = '\n';
  return parse_edge_text(buf.data(), (size_t)sz, matrix_market, zero_indexed,
                         src, dst, n_out, msg);
}

}  // namespace wetric

extern "C" {

int wetric_parse_file(const char *path, int matrix_market, int zero_indexed,
                      uint32_t **src, uint32_t **dst, uint64_t *count,
                      uint64_t *n) {
  if (!path || !src || !dst || !count || !n) return WETRIC_EINVAL;
  std::vector<uint32_t> s, d;
  std::string msg;
  const int st = wetric::parse_edge_file(path, matrix_market != 0,
                                         zero_indexed != 0, &s, &d, n, &msg);
  if (st != WETRIC_OK) return st;
  const size_t bytes = (s.size() ? s.size() : 1) * sizeof(uint32_t);
  *src = (uint32_t *)malloc(bytes);
  *dst = (uint32_t *)malloc(bytes);
  if (!*src || !*dst) {
    free(*src);
    free(*dst);
    *src = *dst = nullptr;
    return WETRIC_ENOMEM;
  }
  if (!s.empty()) {
    memcpy(*src, s.data(), s.size() * sizeof(uint32_t));
    memcpy(*dst, d.data(), d.size() * sizeof(uint32_t));
  }
  *count = s.size();
  return WETRIC_OK;
}

void wetric_free_buffer(void *p) { free(p); }

}  // extern "C"
