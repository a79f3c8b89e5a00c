// preprocess.cuh -- device preprocessing entry points (see preprocess.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace wetric {

// A CSR held in library-owned device memory: row_ptr u64[n+1], col_ind
// u32[m].
struct DeviceCsr {
  DeviceContext *ctx = nullptr;
  cudaStream_t stream = nullptr;
  uint64_t n = 0, m = 0;
  uint64_t *row_ptr = nullptr;
  uint32_t *col_ind = nullptr;
  void release();
  ~DeviceCsr() { release(); }
};

// Raw pairs (0-based ids, device buffers) -> oriented CSR: the combined
// work of read_graph + preprocess (tc.cu:561-787). n_hint == 0 takes
// n = max id over non-loop pairs + 1 (tc.cu:625).
// With group_base (device u64[G+1]) the pairs are a disjoint union of G
// graphs, graph g owning ids [group_base[g], group_base[g+1]); vertices are
// then ranked inside their own graph, so each graph keeps its id range and
// gets exactly the CSR it would get alone (shifted by group_base[g]).
int orient_pairs(DeviceContext *ctx, cudaStream_t st, const uint32_t *src,
                 const uint32_t *dst, uint64_t P, uint64_t n_hint,
                 DeviceCsr *out, const uint64_t *group_base = nullptr,
                 uint32_t G = 0);

// Raw pairs -> symmetric deduplicated CSR without self-loops (the CSR that
// read_graph returns, tc.cu:561-685).
int symmetric_from_pairs(DeviceContext *ctx, cudaStream_t st,
                         const uint32_t *src, const uint32_t *dst, uint64_t P,
                         uint64_t n_hint, DeviceCsr *out);

// CSR (device) -> oriented CSR, following preprocess (tc.cu:687-787):
// degree = row length, stable ascending-degree rank, keep (v, w) as
// (rank v, rank w) when rank w > rank v, rows sorted.
int orient_csr(DeviceContext *ctx, cudaStream_t st, const uint64_t *rp,
               const uint32_t *ci, uint64_t n, uint64_t m, DeviceCsr *out);

}  // namespace wetric
