// csr_cache.cpp -- binary CSR cache: a CSR written once (after the text
// parse and the preprocessing) and read back without parsing.
//
// The reference re-parses its text input on every run (tc.cu:561-685);
// parsing a large Matrix Market file costs far more than counting it. The
// cache stores a CSR as it is in memory:
//
//   bytes 0-7    magic "WTRCSR01"
//   bytes 8-15   n (u64)          bytes 16-23  m (u64)
//   bytes 24-27  flags (u32: the wetric_csr ORIENTED / SYMMETRIC bits)
//   bytes 28-31  offset width (u32, 8)
//   then row_ptr as u64[n+1], then col_ind as u32[m] (little-endian host
//   order, the order of every B200 host).
//
// Loading checks the header against the file size and the CSR itself
// (row_ptr starts at 0, never decreases and ends at m; every column < n),
// so a truncated or foreign file is an error, never a wrong count.
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/wetric.h"

namespace {

const char kMagic[8] = {'W', 'T', 'R', 'C', 'S', 'R', '0', '1'};

struct Header {
  char magic[8];
  uint64_t n, m;
  uint32_t flags, offset_bytes;
};
static_assert(sizeof(Header) == 32, "cache header is 32 bytes");

struct File {
  FILE *f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

}  // namespace

extern "C" {

int wetric_save_csr(const char *path, const wetric_csr *csr) {
  if (!path || !csr || (csr->n > 0 && !csr->row_ptr) ||
      (csr->m > 0 && !csr->col_ind))
    return WETRIC_EINVAL;
  if (csr->flags & WETRIC_CSR_DEVICE) return WETRIC_EINVAL;  // host buffers only
  const uint64_t n = csr->n, m = csr->m;
  File out;
  out.f = fopen(path, "wb");
  if (!out.f) return WETRIC_EIO;
  Header h;
  memcpy(h.magic, kMagic, 8);
  h.n = n;
  h.m = m;
  h.flags = csr->flags & (WETRIC_CSR_ORIENTED | WETRIC_CSR_SYMMETRIC);
  h.offset_bytes = 8;
  if (fwrite(&h, sizeof(h), 1, out.f) != 1) return WETRIC_EIO;
  if (csr->flags & WETRIC_CSR_OFFSETS32) {
    // widen in chunks so no second copy of the offsets is needed
    const uint32_t *rp = static_cast<const uint32_t *>(csr->row_ptr);
    uint64_t chunk[4096];
    for (uint64_t i = 0; i <= n; i += 4096) {
      const uint64_t k = (n + 1 - i) < 4096 ? (n + 1 - i) : 4096;
      for (uint64_t j = 0; j < k; ++j) chunk[j] = rp[i + j];
      if (fwrite(chunk, 8, k, out.f) != k) return WETRIC_EIO;
    }
  } else if (fwrite(csr->row_ptr, 8, n + 1, out.f) != n + 1) {
    return WETRIC_EIO;
  }
  if (m > 0 && fwrite(csr->col_ind, 4, m, out.f) != m) return WETRIC_EIO;
  if (fclose(out.f) != 0) {
    out.f = nullptr;
    return WETRIC_EIO;
  }
  out.f = nullptr;
  return WETRIC_OK;
}

int wetric_load_csr(const char *path, wetric_csr *csr) {
  if (!path || !csr) return WETRIC_EINVAL;
  memset(csr, 0, sizeof(*csr));
  File in;
  in.f = fopen(path, "rb");
  if (!in.f) return WETRIC_EIO;
  Header h;
  if (fread(&h, sizeof(h), 1, in.f) != 1 || memcmp(h.magic, kMagic, 8) != 0 ||
      h.offset_bytes != 8 || h.n >= (1ull << 32) || h.m > (1ull << 40))
    return WETRIC_EIO;
  if (fseek(in.f, 0, SEEK_END) != 0) return WETRIC_EIO;
  const long long size = ftell(in.f);
  const unsigned long long want =
      sizeof(Header) + (h.n + 1) * 8ull + h.m * 4ull;
  if (size < 0 || (unsigned long long)size != want) return WETRIC_EIO;
  if (fseek(in.f, (long)sizeof(Header), SEEK_SET) != 0) return WETRIC_EIO;
  uint64_t *rp = (uint64_t *)malloc((h.n + 1) * 8);
  uint32_t *ci = (uint32_t *)malloc((h.m ? h.m : 1) * 4);
  if (!rp || !ci) {
    free(rp);
    free(ci);
    return WETRIC_ENOMEM;
  }
  bool ok = fread(rp, 8, h.n + 1, in.f) == h.n + 1 &&
            (h.m == 0 || fread(ci, 4, h.m, in.f) == h.m);
  // the CSR itself: offsets from 0 to m without decreasing, columns < n
  ok = ok && rp[0] == 0 && rp[h.n] == h.m;
  for (uint64_t v = 0; ok && v < h.n; ++v) ok = rp[v] <= rp[v + 1];
  for (uint64_t j = 0; ok && j < h.m; ++j) ok = ci[j] < h.n;
  if (!ok) {
    free(rp);
    free(ci);
    return WETRIC_EIO;
  }
  csr->n = h.n;
  csr->m = h.m;
  csr->row_ptr = rp;
  csr->col_ind = ci;
  csr->flags = h.flags;
  return WETRIC_OK;
}

}  // extern "C"
