/*
 * wetric.h -- C ABI of the B200-native wedge-parallel triangle counter.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and never
 * calls exit(): failures come back as a status code (or a sentinel return
 * value plus wetric_last_error()).
 *
 * Two groups of entry points:
 *
 *  1. Drop-in mirrors of the reference's own functions (same struct layouts,
 *     same argument meaning), so an existing caller of the reference's
 *     count path can switch by renaming calls:
 *       wetric_read_graph      <- read_graph   (tc.cu:561)
 *       wetric_preprocess      <- preprocess   (tc.cu:687)
 *       wetric_tc_gpu          <- tc_GPU       (tc.cu:315)
 *       wetric_free_graph      <- free_graph   (tc.cu:789)
 *       wetric_*_big_graph / wetric_tc_gpu_big <- experiments/tc_big_graphs.cu
 *                                  (BIG_GRAPH_TYPE, tc_GPU at :315)
 *
 *  2. The library interface: wetric_count / wetric_count_ex over a
 *     wetric_csr (u64 offsets, host or device buffers), device-side
 *     preprocessing of raw edge lists, and a context for batched counting.
 *
 * All device work runs on one CUDA device per call (device 0 unless
 * wetric_opts.device says otherwise), on sm_100a kernels.
 *
 * Device memory: scratch comes from the device's default stream-ordered
 * pool (cudaMallocAsync). The first call that uses a device sets its pool
 * to keep freed memory for the life of the process and grows it once by
 * 4 GiB (allocated and freed at once), so later counts take their scratch
 * without asking the driver for memory. That memory stays with the pool:
 * other allocators in the process (a framework's caching allocator) see
 * that much less free memory. If the 4 GiB cannot be had, the pool grows
 * on demand instead. wetric_count_noalloc never touches the pool.
 */
#ifndef WETRIC_H
#define WETRIC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */

/* The reference exits the process on every error (tc.cu:46-54, 299-304,
 * 397-400); these codes replace those exits. */
enum {
  WETRIC_OK = 0,
  WETRIC_EINVAL = 1,    /* bad argument: a % 32 != 0, s == 0, unsorted or
                           unoriented CSR when validation is on, NULL ptr  */
  WETRIC_ENOMEM = 2,    /* device/host allocation failed or the context's
                           HBM budget would be exceeded                    */
  WETRIC_ETIMEDOUT = 3, /* a bounded device-side wait ran out               */
  WETRIC_ECUDA = 4,     /* a CUDA runtime call failed                       */
  WETRIC_ERANGE = 5,    /* sizes beyond the limits (n >= 2^32, d+ >= 2^30)  */
  WETRIC_EIO = 6,       /* graph file missing, unreadable or malformed      */
  WETRIC_ENODEV = 7,    /* no CUDA device                                   */
  WETRIC_EBUSY = 8      /* context queue full / ticket not finished         */
};

/* Status of the last failing call on this host thread (0 if none). */
int wetric_last_error(void);
/* Static, human-readable text for a status code. */
const char *wetric_strerror(int status);
/* Message with detail for the last failing call on this host thread. */
const char *wetric_last_error_message(void);

/* ------------------------------------------- reference-compatible mirrors */

/* Same layout as GRAPH_TYPE (tc.cu:58-63): u32 offsets. */
typedef struct {
  uint32_t numVertices;
  uint32_t numEdges;
  uint32_t *rowPtr;
  uint32_t *colInd;
} wetric_graph;

/* Same layout as BIG_GRAPH_TYPE (experiments/tc_big_graphs.cu:58-63). */
typedef struct {
  uint32_t numVertices;
  uint64_t numEdges;
  uint64_t *rowPtr;
  uint32_t *colInd;
} wetric_big_graph;

/* Same layout as GPU_time (tc.cu:76-79); milliseconds are ADDED to each. */
typedef struct {
  double copy;
  double exec;
} wetric_gpu_time;

/* preprocess_t (tc.cu:56). All three styles run the device pipeline; the
 * value is accepted for CLI compatibility. The vertex order is the stable
 * ascending-degree order of styles 1 and 2 (CUB's stable radix sort in the
 * reference); style 0's qsort tie order is not reproduced (counts agree). */
enum { WETRIC_PREPROCESS_CPU = 0, WETRIC_PREPROCESS_GPU = 1,
       WETRIC_PREPROCESS_GPU_CONSTRAINED = 2 };

/* Replaces read_graph (tc.cu:561-685). Parses a text edge list (mm == 0) or
 * a Matrix Market file (mm != 0): leading lines whose first character is
 * not a digit are skipped; for Matrix Market one more (size) line is
 * skipped; each following line gives "v w" (any further columns on the line
 * are ignored); ids are 1-based unless zero_indexed, and a zero id without
 * zero_indexed is an error (tc.cu:599-602). Self-loops are dropped, both
 * directions are kept, duplicates removed; n = max id + 1 (tc.cu:625).
 * Returns a malloc'd symmetric CSR (free with wetric_free_graph) or NULL
 * with wetric_last_error() set. Dedup runs on the GPU. */
wetric_graph *wetric_read_graph(const char *filename, int matrix_market,
                                int zero_indexed, int preprocess_style);
/* As above with u64 offsets (experiments/tc_big_graphs.cu:567). */
wetric_big_graph *wetric_read_big_graph(const char *filename, int matrix_market,
                                        int zero_indexed, int preprocess_style);

/* Replaces preprocess (tc.cu:687-787): relabels vertices by stable
 * ascending degree, keeps each edge once as (v -> w) with new id w > v, and
 * sorts every row. Runs on the GPU. Returns a malloc'd oriented CSR. */
wetric_graph *wetric_preprocess(const wetric_graph *original_graph,
                                int preprocess_style);
wetric_big_graph *wetric_preprocess_big(const wetric_big_graph *original_graph,
                                        int preprocess_style);

/* Replaces free_graph (tc.cu:789-793). NULL is a no-op. */
void wetric_free_graph(wetric_graph *graph);
void wetric_free_big_graph(wetric_big_graph *graph);

/* Replaces tc_GPU (tc.cu:315-441): counts the triangles of a host-resident
 * oriented CSR (the output of wetric_preprocess) with spread `spread` (> 0)
 * and bitmap length `adjacency_matrix_len` (multiple of 32). Adds the time
 * of the host->device copies to t->copy and of all device work (wedge
 * prefix, bitmap build and count kernels) to t->exec, in milliseconds.
 * Returns UINT64_MAX on error (wetric_last_error() says why); t may be NULL. */
uint64_t wetric_tc_gpu(const wetric_graph *graph, uint32_t spread,
                       uint32_t adjacency_matrix_len, wetric_gpu_time *t);
/* Replaces the big-graph tc_GPU (experiments/tc_big_graphs.cu:315-447). */
uint64_t wetric_tc_gpu_big(const wetric_big_graph *graph, uint32_t spread,
                           uint32_t adjacency_matrix_len, wetric_gpu_time *t);

/* ---------------------------------------------------- library interface */

/* CSR flags. */
#define WETRIC_CSR_ORIENTED  0x1u  /* rows sorted, every col_ind[j] > row,
                                      no duplicates (the output contract of
                                      preprocess, tc.cu:740-787)            */
#define WETRIC_CSR_SYMMETRIC 0x2u  /* raw symmetric adjacency: the library
                                      orients it on the device first        */
#define WETRIC_CSR_DEVICE    0x4u  /* row_ptr / col_ind are device pointers
                                      on opts->device                       */
#define WETRIC_CSR_OFFSETS32 0x8u  /* row_ptr is uint32_t[n+1] instead of
                                      uint64_t[n+1]                         */

typedef struct {
  uint64_t n;            /* vertices                                   */
  uint64_t m;            /* entries of col_ind                         */
  const void *row_ptr;   /* uint64_t[n+1] (uint32_t with OFFSETS32)    */
  const uint32_t *col_ind;
  uint32_t flags;
} wetric_csr;

/* Binary CSR cache (no reference counterpart: the reference re-parses its
 * text input every run, tc.cu:561-685). wetric_save_csr writes a host CSR
 * (u64 or u32 offsets; the ORIENTED / SYMMETRIC flags are kept) to `path`;
 * wetric_load_csr reads it back into host buffers -- row_ptr as
 * uint64_t[n+1], col_ind as uint32_t[m] -- that the caller releases with
 * wetric_free_buffer, after checking the file against its header and the
 * CSR itself. Errors: WETRIC_EINVAL (bad argument, device buffers),
 * WETRIC_EIO (unreadable, truncated or not a cache), WETRIC_ENOMEM. */
int wetric_save_csr(const char *path, const wetric_csr *csr);
int wetric_load_csr(const char *path, wetric_csr *csr);
/* Releases a host buffer the library allocated (wetric_load_csr,
 * wetric_parse_file). */
void wetric_free_buffer(void *p);

typedef struct {
  uint32_t spread;        /* wedges per thread per tile (s > 0)            */
  uint32_t bitmap_len;    /* a: bitmap over the last a vertices (a % 32 == 0) */
  uint32_t block;         /* threads per block: 0 = library default       */
  uint32_t validate;      /* != 0: check the ORIENTED contract on device  */
  uint64_t wedge_begin;   /* count only wedges [wedge_begin, wedge_end);  */
  uint64_t wedge_end;     /*   wedge_end == 0 means "to the end"          */
  int32_t device;         /* CUDA device ordinal                          */
  uint32_t l2_persist;    /* != 0: pin the bitmap in L2 (access window)   */
  uint32_t kernel;        /* count kernel: 0 = default (8), 1 = block-tile,
                             2 = warp-staged, 3 = row-walk with the
                             shared-memory stage, 4 = row-walk, 5 = 4 at
                             6 blocks/SM, 6 = 5 with per-row hash sets
                             for rows outside the bitmap, 7 = 6 with
                             long-row segments (row-uniform checks),
                             8 = 7 with 16-bit near hash sets for the
                             rows within 65536 ids of the last vertex   */
  uint32_t opt_flags;     /* WETRIC_OPT_* bits                            */
  void *stream;           /* cudaStream_t, NULL = library stream          */
  uint32_t core_len;      /* dense core (kernels 7, 8): the top core_len
                             vertices of the degree order, whose
                             out-neighbours all lie in the same top range,
                             have their wedges counted by row ANDs of a
                             core bit matrix instead of one edge check per
                             wedge. 0 = sized by the library from the row
                             offsets (at most 65536, or none when the top
                             rows are too sparse to pay); WETRIC_CORE_OFF =
                             no core; else that many (capped at 65536).
                             The count does not depend on it.            */
  uint32_t shell_len;     /* with a core that covers the bitmap's rows:
                             the shell_len vertices below the core count
                             each pair (v, w) the cheaper way -- a row AND
                             when w is a core vertex and that reads fewer
                             words than the pair has wedges, else the
                             usual edge checks. 0 or WETRIC_CORE_OFF = no
                             shell (the default: on R-MAT scale 22 the
                             wedge-check kernel handles those vertices
                             faster).                                     */
} wetric_opts;

#define WETRIC_CORE_OFF 0xFFFFFFFFu

/* Keep u64 row offsets in the count even when m < 2^32 (by default they
 * are narrowed to u32, which halves the offset bytes of every check). */
#define WETRIC_OPT_KEEP_U64_OFFSETS 0x1u
/* Launch the row-walk count kernels (3-8) with one warp per tile instead
 * of a persistent grid, so work on other streams gets SMs as the count's
 * blocks finish (the serving lanes use this). */
#define WETRIC_OPT_ONE_PASS 0x2u
/* No pair streams for short rows. By default a whole-graph count (kernel
 * 8, 32-bit offsets, columns not copied in row chunks) counts each vertex
 * with d+ <= 64 whose neighbours' rows are short too the other way round:
 * its out-neighbours go into a shared-memory set and the rows of those
 * neighbours stream through it (k_count_pairs), instead of one set lookup
 * per wedge. The count is the same either way. */
#define WETRIC_OPT_NO_PAIR_STREAMS 0x4u

typedef struct {
  double copy_ms;         /* host->device copies of the CSR (host input
                             of 2^22+ columns: the row offsets' copy plus
                             the column chunks', which overlap the count) */
  double prep_ms;         /* device orientation (SYMMETRIC input only)    */
  double exec_ms;         /* wedge prefix + bitmap + count kernels        */
  double count_ms;        /* the count kernels alone: the wedge-check,
                             dense-core and shell kernels (summed
                             over the row-chunk launches of a chunked
                             host input)                                  */
  uint64_t n, m;          /* of the oriented graph                        */
  uint64_t wedges;        /* W = sum over v of C(d+(v), 2)                */
  uint64_t wedges_counted;/* wedges in [wedge_begin, wedge_end)           */
  uint64_t max_out_degree;
  uint32_t spread, bitmap_len, block, grid;
  uint32_t launches;      /* kernels launched by this call                */
  uint32_t core_len;      /* dense core vertices used (0: none)           */
  uint64_t core_wedges;   /* wedges counted by the core kernel            */
  double core_ms;         /* the core kernel alone (part of count_ms)     */
  uint64_t shell_len;     /* shell vertices used (0: none)                */
  uint64_t shell_wedges;  /* wedges counted by the shell kernel           */
  double shell_ms;        /* the shell kernel alone (part of count_ms)    */
  uint64_t pair_rows;     /* vertices counted by pair streams (0: none)   */
  uint64_t pair_wedges;   /* their wedges (part of wedges_counted)        */
  double pair_ms;         /* the pair-stream kernel alone (part of
                             count_ms)                                    */
} wetric_stats;

/* Cap the device memory this library may hold on `device` (0 = no cap).
 * Allocations beyond it fail with WETRIC_ENOMEM before reaching the driver;
 * serving admission and fault tests use it. */
int wetric_set_hbm_budget(int device, uint64_t bytes);

/* Fill opts with defaults (s = 5, a = 8192, device 0, whole wedge range). */
void wetric_opts_init(wetric_opts *opts);

/* Exact triangle count of a CSR with spread s and bitmap length a, on
 * device 0. Returns UINT64_MAX on error (see wetric_last_error()). This is
 * tc_GPU (tc.cu:315) generalised to u64 offsets, host or device buffers and
 * symmetric or oriented input. */
uint64_t wetric_count(const wetric_csr *csr, uint32_t s, uint32_t a);

/* Status-returning form with options and statistics (stats may be NULL).
 * With a wedge range it counts the triangles closed by the wedges of that
 * range only: summing disjoint ranges that cover [0, W) gives the count. */
int wetric_count_ex(const wetric_csr *csr, const wetric_opts *opts,
                    uint64_t *count, wetric_stats *stats);

/* Total wedges W and max out-degree of an ORIENTED csr (device work). */
int wetric_wedge_total(const wetric_csr *csr, int device, uint64_t *wedges,
                       uint64_t *max_out_degree);

/* Algorithmic bytes of the wedge-check count on an ORIENTED csr: rows,
 * columns and wedge prefix read once (8(n+1) + 4m + 8(n+1)) plus, for
 * every wedge with middle vertex w, 4 + 16 + 4*ceil(log2(d+(w) + 1)). */
int wetric_algorithmic_bytes(const wetric_csr *csr, int device,
                             uint64_t *bytes);

/* Device preprocessing of a raw edge list (the work of read_graph +
 * preprocess, tc.cu:561-787, on the GPU): pairs (src[i], dst[i]), 0-based
 * ids; self-loops dropped; direction and duplicates ignored. Produces the
 * oriented CSR in device memory owned by the returned handle.
 * `flags` may hold WETRIC_CSR_DEVICE when src/dst are device pointers.
 * n_hint: 0 = n from max id + 1 over non-loop pairs, else use n_hint
 * (ids must be < n_hint). */
typedef struct wetric_oriented_s *wetric_oriented;
int wetric_orient_edges(const uint32_t *src, const uint32_t *dst,
                        uint64_t num_pairs, uint64_t n_hint, uint32_t flags,
                        int device, wetric_oriented *out, wetric_stats *stats);
/* A CSR view of the handle's device arrays (flags ORIENTED|DEVICE). */
int wetric_oriented_csr(wetric_oriented h, wetric_csr *csr);
/* Copy the oriented CSR to host buffers (uint64_t[n+1], uint32_t[m]). */
int wetric_oriented_download(wetric_oriented h, uint64_t *row_ptr,
                             uint32_t *col_ind);
void wetric_oriented_free(wetric_oriented h);

/* ------------------------------------------------- count without allocation */

/* No counterpart in the reference. For callers that cannot allocate device
 * memory when they count -- code running inside another framework's memory
 * pool or under a hard device-memory quota, hosts that forbid allocation
 * after start-up, threads that must not take the driver's allocation locks.
 * Counts an ORIENTED device CSR (WETRIC_CSR_DEVICE | WETRIC_CSR_ORIENTED,
 * optionally WETRIC_CSR_OFFSETS32) like wetric_count_ex, but every scratch
 * buffer comes from one static device array of WETRIC_NOALLOC_SCRATCH_BYTES
 * that each GPU loading the library holds until the process exits; nothing
 * is allocated or freed. Limits: n <= WETRIC_NOALLOC_MAX_VERTICES,
 * a <= WETRIC_NOALLOC_MAX_BITMAP_LEN, and the tile map (W / (256 s) entries)
 * must fit the rest of the array; larger inputs return WETRIC_ERANGE.
 * The first call on a device looks up the array's device address (with
 * that device current) and caches it with the id of the device's context;
 * a call in a new context of the device (after cudaDeviceReset) looks it
 * up again. Make that first call before any stream capture. Calls share the
 * array and it keeps the last call's contents (each call clears what must
 * start at zero); calls that overlap on the GPU race, so order them.
 * Runs on `stream` (NULL = the default stream) and waits for the result. */
#define WETRIC_NOALLOC_SCRATCH_BYTES (64u << 20)
#define WETRIC_NOALLOC_MAX_VERTICES 1000000u
#define WETRIC_NOALLOC_MAX_BITMAP_LEN 8192u
int wetric_count_noalloc(const wetric_csr *csr, uint32_t s, uint32_t a,
                         int device, void *stream, uint64_t *count);

/* ------------------------------------------------------ batched counting */

/* Many graphs of uneven sizes counted together (no reference counterpart:
 * the reference counts one graph per run, tc.cu:896-913). The batch is
 * preprocessed once on the device as a disjoint union in which every graph
 * keeps its own id range and its own degree order (so each graph's oriented
 * CSR equals the one it gets alone), stays resident, and is counted by a
 * persistent kernel that pulls (graph, wedge-range) tiles from a device work
 * counter; the launches are captured in a CUDA graph and replayed. */
typedef struct wetric_batch_s *wetric_batch;

typedef struct {
  uint32_t spread;         /* s for every graph; 0 = tuned per graph size   */
  uint32_t bitmap_len;     /* per-graph bitmap over min(a, n_g) vertices    */
  uint32_t use_cuda_graph; /* != 0: capture the count and replay it         */
  uint32_t autotune;       /* != 0 (and spread == 0): time candidate spreads
                              for each size/skew bucket of graphs not yet in
                              this device's tuning table, and use the table */
  uint64_t bitmap_cap_bytes; /* total bitmap memory (0 = 2 GiB)             */
  uint32_t no_pair_streams;  /* != 0: no pair streams for the short rows
                                (WETRIC_OPT_NO_PAIR_STREAMS for a batch)   */
} wetric_batch_opts;

void wetric_batch_opts_init(wetric_batch_opts *opts);

/* Graph g owns pairs [pair_off[g], pair_off[g+1]) of src/dst, 0-based ids
 * below n[g] (pair_off, n: host arrays of G+1 and G entries; src/dst host
 * or, with WETRIC_CSR_DEVICE in flags, device pointers). Self-loops are
 * dropped and duplicates merged per graph. The sum of n[g] must be < 2^32. */
int wetric_batch_create(const uint32_t *src, const uint32_t *dst,
                        const uint64_t *pair_off, const uint64_t *n,
                        uint32_t G, uint32_t flags, int device,
                        const wetric_batch_opts *opts, wetric_batch *out);
/* counts: host uint64_t[G]; stats (may be NULL): exec_ms = device time of
 * the count, wedges = W of the whole batch, launches = kernels per count. */
int wetric_batch_count(wetric_batch b, uint64_t *counts, wetric_stats *stats);
/* Per-graph W and oriented edge counts (host arrays of G entries; either
 * may be NULL). */
int wetric_batch_info(wetric_batch b, uint64_t *wedges, uint64_t *edges);
/* The spread s_g each graph is counted with (host array of G entries):
 * tiles of 256 * s_g wedges. */
int wetric_batch_spreads(wetric_batch b, uint32_t *spread);
void wetric_batch_free(wetric_batch b);

/* --------------------------------------------------------------- serving */

/* A counting service (no reference counterpart: the reference counts one
 * file per run). Requests -- one graph each, given as raw pairs -- may be
 * submitted at any time from any thread. They go to one of two lanes by
 * size (large_pairs), so small graphs never wait behind large ones; the two
 * lanes run on their own streams and overlap on the device. A lane's worker
 * takes its waiting requests in arrival order while their device footprint
 * fits the (shared) HBM budget.
 *   resident (default): the worker preprocesses each request while the
 *     resident counting kernel runs, then folds its tiles into that
 *     kernel's work queue; a large request is fed in items of item_tiles
 *     tiles so later small ones interleave with it;
 *   otherwise: one request runs the single-graph path, several run as one
 *     batch (one preprocessing pass, one count launch), and requests that
 *     arrive meanwhile join the lane's next batch.
 * A request's src/dst buffers are borrowed until its ticket completes. */
typedef struct wetric_server_s *wetric_server;

typedef struct {
  uint64_t hbm_budget;       /* admission cap on device bytes (0 = 150 GiB) */
  uint64_t max_batch_pairs;  /* pairs folded into one batch (0 = 2^30)      */
  uint32_t max_batch_graphs; /* graphs folded into one batch (0 = 4096)     */
  uint32_t spread;           /* s (0 = 5)                                   */
  uint32_t bitmap_len;       /* per-graph bitmap cap a (multiple of 32)     */
  uint32_t queue_capacity;   /* waiting requests before EBUSY (0 = 65536)   */
  uint64_t large_pairs;      /* requests with at least this many pairs go to
                                the large lane (own thread and stream);
                                0 = one lane for all (init: 8 Mi pairs)    */
  uint64_t reserve_bytes;    /* device memory each lane's stream reserves in
                                the pool at creation (init: 8 GiB, at most
                                half the budget), so serving does not grow
                                the pool                                   */
  uint32_t resident;         /* 0 (init): each lane batches its waiting
                                requests and counts them with its own
                                launches; != 0: one resident counting
                                kernel stays on the device and takes the
                                tiles of every request as soon as it is
                                preprocessed (requests are folded into the
                                running kernel's work queue). On the
                                Poisson serving workload the lanes measured
                                p50 2.5 ms / p99 82 ms against 17.7 / 403 ms
                                resident, so they are the default.          */
  uint32_t item_tiles;       /* resident: a request with more tiles is fed
                                to the queue in items of this many tiles (at
                                most 64 items a request), a few items ahead
                                of the kernel, so smaller requests published
                                meanwhile are not stuck behind it
                                (init: 65536)                              */
} wetric_server_opts;

typedef struct {
  uint64_t completed, failed, batches, waiting, admitted_bytes;
  double mean_batch_graphs; /* graphs per counted batch                   */
  double p50_ms, p99_ms;    /* submit-to-completion latency               */
  double count_busy_ms;     /* device time spent in batch counts          */
  double admit_busy_ms;     /* wall time spent building batches           */
  uint64_t pairs_admitted;  /* input pairs folded into batches            */
  double queue_p50_ms;      /* submit until a lane worker takes it        */
  double small_p50_ms, small_p99_ms; /* latency in the small lane          */
  double large_p50_ms, large_p99_ms; /* latency in the large lane          */
  uint64_t large_completed; /* requests completed by the large lane       */
  uint64_t resident_launches; /* launches of the resident kernel (it ends
                                 after a short idle period)               */
  uint64_t recycles;        /* resident: drains that freed retired memory */
  uint32_t resident_last_exit; /* how the last resident kernel ended: 0 =
                                  still running, 1 = stopped, 2 = gave up
                                  waiting on an empty queue (its bounded
                                  wait ran out)                            */
  uint32_t launch_error_code; /* cudaError_t of the last failed launch of
                                  the resident kernel (0: none)           */
  /* resident queue state (diagnostics): requests registered with the kernel
   * and not yet completed, those of them still being fed, queue items
   * published and taken by the kernel, 1 while draining for a recycle,
   * failed launches of the resident kernel, and each lane's phase (0 =
   * waiting for a request or for admission, 1 = preprocessing, 2 = waiting
   * for queue space, 3 = publishing) */
  uint64_t live, feeding, items_published, items_taken;
  uint32_t draining, launch_errors;
  uint32_t lane_phase[2];
} wetric_server_stats;

void wetric_server_opts_init(wetric_server_opts *opts);
int wetric_server_create(int device, const wetric_server_opts *opts,
                         wetric_server *out);
/* 0-based pairs with ids < n (host, or device with WETRIC_CSR_DEVICE in
 * flags). Returns WETRIC_EBUSY when the queue is full. */
int wetric_server_submit(wetric_server s, const uint32_t *src,
                         const uint32_t *dst, uint64_t pairs, uint64_t n,
                         uint32_t flags, uint64_t *ticket);
/* The same for a graph given as a CSR (ORIENTED or SYMMETRIC, host or
 * device, u64 or WETRIC_CSR_OFFSETS32 offsets, n <= 2^32): the server
 * copies it into pairs of its own before returning, so the caller's
 * buffers are free at once. The count is the graph's, whatever its ids'
 * order (the server orients it itself). */
int wetric_server_submit_csr(wetric_server s, const wetric_csr *csr, uint64_t *ticket);
/* WETRIC_EBUSY while the ticket is pending; on completion the ticket is
 * consumed and *count / *latency_ms are set. */
int wetric_server_poll(wetric_server s, uint64_t ticket, uint64_t *count,
                       double *latency_ms);
/* Blocks up to timeout_ms; WETRIC_ETIMEDOUT if still pending. */
int wetric_server_wait(wetric_server s, uint64_t ticket, uint32_t timeout_ms,
                       uint64_t *count, double *latency_ms);
int wetric_server_get_stats(wetric_server s, wetric_server_stats *out);
/* Stops admitting, finishes admitted work, fails requests still waiting
 * (WETRIC_EBUSY), joins the threads. */
void wetric_server_destroy(wetric_server s);

#ifdef __cplusplus
}
#endif

#endif /* WETRIC_H */
