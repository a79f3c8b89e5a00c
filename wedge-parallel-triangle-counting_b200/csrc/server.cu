// server.cu -- a counting service: requests (one graph each) arrive at any
// time, are admitted against an HBM budget, preprocessed and counted, in
// batches when several are waiting, while other requests are on the device.
//
// The reference has no serving layer (one graph per process run,
// tc.cu:816-918). Requests go to one of two lanes by size (pairs below
// opts.large_pairs: the small lane; the rest: the large lane), so a small
// graph never waits behind a large one. Each lane is one worker thread with
// its own CUDA stream (all of a lane's device memory is allocated and freed
// in stream order on that stream; the small lane's stream has the higher
// priority, and counts run one warp per tile, so the lanes interleave). The worker takes the lane's waiting
// requests in arrival order while their estimated footprint fits the
// shared budget, then
//   * one request: the single-graph path (orient_pairs + count_oriented,
//     exactly what a plain call does);
//   * several (small lane only; the large lane takes one at a time): one
//     batch (batch_create: one preprocessing pipeline over the disjoint
//     union; batch_count: one launch of one warp per tile, so the other
//     lane's blocks get SMs as they finish),
// completes the tickets and releases the memory. Requests that arrive while
// a lane is busy are folded into its next batch (continuous batching); the
// two lanes overlap on the device.
// Input buffers are borrowed until the request completes.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/wetric.h"
#include "batch.cuh"
#include "common.cuh"
#include "count.cuh"
#include "preprocess.cuh"

namespace wetric {

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t ticket = 0;
  const uint32_t *src = nullptr, *dst = nullptr;
  uint64_t pairs = 0, n = 0;
  bool on_device = false;
  Clock::time_point arrived;
  uint64_t bytes = 0;  // admission estimate
  bool solo = false;   // re-admitted alone after its batch failed
};

struct Result {
  bool done = false;
  int status = WETRIC_OK;
  uint64_t count = 0;
  double latency_ms = 0.0;
};

}  // namespace

struct Server;

struct Lane {
  Server *srv = nullptr;
  cudaStream_t stream = nullptr;
  std::deque<Request> waiting;
  std::thread worker;
};

struct Server {
  DeviceContext *ctx = nullptr;
  wetric_server_opts opt{};
  std::mutex mu;
  std::condition_variable cv_admit, cv_done;
  Lane lanes[2];  // 0: small requests, 1: large requests
  std::unordered_map<uint64_t, Result> results;
  uint64_t next_ticket = 1;
  uint64_t admitted_bytes = 0;
  bool stop = false;
  // statistics
  uint64_t completed = 0, batches = 0, failed = 0, graphs_in_batches = 0;
  std::vector<double> latencies, lane_latencies[2], queue_ms;
  double busy_ms = 0.0;   // device time of the counts
  double admit_ms = 0.0;  // wall time of preprocessing
  uint64_t pairs_admitted = 0;
  size_t waiting_total() const {
    return lanes[0].waiting.size() + lanes[1].waiting.size();
  }
};

namespace {

// Device bytes a request holds while being preprocessed: its pairs copied
// into the union (8 B/pair), canonical keys and sort buffers (16 B/pair),
// orientation keys (16 B/pair), the CSR (4 B/pair + 8 B/vertex), the
// per-row hash sets (at most 16 B/pair) and the per-vertex work arrays
// (about 40 B/vertex).
uint64_t estimate_bytes(uint64_t pairs, uint64_t n) {
  return 60 * pairs + 48 * n + (1u << 20);
}

// One request through the single-graph path on the lane's stream.
int run_single(Server *s, Lane *ln, const Request &r, uint64_t *count,
               double *prep_ms, double *count_ms) {
  const cudaStream_t st = ln->stream;
  const Clock::time_point t0 = Clock::now();
  Scratch<uint32_t> us, ud;
  const uint32_t *src = r.src, *dst = r.dst;
  if (!r.on_device && r.pairs) {
    WETRIC_TRY(us.alloc(s->ctx, st, r.pairs));
    WETRIC_TRY(ud.alloc(s->ctx, st, r.pairs));
    WETRIC_CUDA_TRY(cudaMemcpyAsync(us.ptr, r.src, r.pairs * 4,
                                    cudaMemcpyHostToDevice, st));
    WETRIC_CUDA_TRY(cudaMemcpyAsync(ud.ptr, r.dst, r.pairs * 4,
                                    cudaMemcpyHostToDevice, st));
    src = us.ptr;
    dst = ud.ptr;
  }
  DeviceCsr csr;
  WETRIC_TRY(orient_pairs(s->ctx, st, src, dst, r.pairs, r.n, &csr));
  us.release();
  ud.release();
  Scratch<uint32_t> narrow;
  CountArgs a;
  a.n = csr.n;
  a.m = csr.m;
  a.row_ptr = csr.row_ptr;
  a.col_ind = csr.col_ind;
  if (csr.m < (1ull << 32) && csr.n > 0) {
    WETRIC_TRY(narrow.alloc(s->ctx, st, csr.n + 1));
    WETRIC_TRY(narrow_offsets(s->ctx, st, csr.row_ptr, csr.n, narrow.ptr));
    a.row_ptr = narrow.ptr;
    a.offsets32 = true;
  }
  a.spread = s->opt.spread ? s->opt.spread : 5;
  a.bitmap_len = s->opt.bitmap_len;
  a.persistent = false;  // the other lane's blocks get SMs as ours end
  WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  *prep_ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
  CountResult cr;
  WETRIC_TRY(count_oriented(s->ctx, st, a, &cr));
  *count = cr.triangles;
  *count_ms = cr.exec_ms;
  return WETRIC_OK;
}

// Several requests as one batch on the lane's stream.
int run_batch(Server *s, Lane *ln, const std::vector<Request> &reqs,
              std::vector<uint64_t> *counts, double *prep_ms,
              double *count_ms) {
  const cudaStream_t st = ln->stream;
  const Clock::time_point t0 = Clock::now();
  const uint32_t G = (uint32_t)reqs.size();
  std::vector<uint64_t> off(G + 1, 0), n(G);
  for (uint32_t g = 0; g < G; ++g) {
    off[g + 1] = off[g] + reqs[g].pairs;
    n[g] = reqs[g].n;
  }
  Scratch<uint32_t> us, ud;
  WETRIC_TRY(us.alloc(s->ctx, st, off[G]));
  WETRIC_TRY(ud.alloc(s->ctx, st, off[G]));
  for (uint32_t g = 0; g < G; ++g) {
    const Request &r = reqs[g];
    if (!r.pairs) continue;
    const cudaMemcpyKind k =
        r.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    WETRIC_CUDA_TRY(cudaMemcpyAsync(us.ptr + off[g], r.src, r.pairs * 4, k, st));
    WETRIC_CUDA_TRY(cudaMemcpyAsync(ud.ptr + off[g], r.dst, r.pairs * 4, k, st));
  }
  BatchOptions bo;
  bo.spread = s->opt.spread ? s->opt.spread : 5;
  bo.bitmap_len = s->opt.bitmap_len;
  bo.use_graph = false;   // each batch is counted once
  bo.persistent = false;  // the other lane's blocks get SMs as ours end
  Batch b;
  WETRIC_TRY(batch_create(s->ctx, us.ptr, ud.ptr, off.data(), n.data(), G,
                          true, bo, &b, st));
  us.release();
  ud.release();
  *prep_ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
  counts->assign(G, 0);
  uint32_t launches = 0;
  WETRIC_TRY(batch_count(&b, counts->data(), count_ms, &launches, st));
  return WETRIC_OK;
}

int warm_up_lane(Server *s, Lane *ln) {
  // K4 (4 triangles) and a triangle, as host pairs
  static const uint32_t k4s[] = {0, 0, 0, 1, 1, 2}, k4d[] = {1, 2, 3, 2, 3, 3};
  static const uint32_t k3s[] = {0, 1, 0}, k3d[] = {1, 2, 2};
  Request a, b;
  a.src = k4s; a.dst = k4d; a.pairs = 6; a.n = 4;
  b.src = k3s; b.dst = k3d; b.pairs = 3; b.n = 3;
  uint64_t c = 0;
  double p = 0, q = 0;
  WETRIC_TRY(run_single(s, ln, a, &c, &p, &q));
  std::vector<uint64_t> counts;
  WETRIC_TRY(run_batch(s, ln, {a, b}, &counts, &p, &q));
  if (c != 4 || counts.size() != 2 || counts[0] != 4 || counts[1] != 1) {
    set_error(WETRIC_ECUDA, "server warm-up counted wrongly");
    return WETRIC_ECUDA;
  }
  uint64_t reserve = s->opt.reserve_bytes;
  if (reserve > s->opt.hbm_budget / 2) reserve = s->opt.hbm_budget / 2;
  if (reserve) {
    Scratch<unsigned char> r;
    if (r.alloc(s->ctx, ln->stream, reserve) != WETRIC_OK) clear_error();
  }
  WETRIC_CUDA_TRY(cudaStreamSynchronize(ln->stream));
  return WETRIC_OK;
}

void lane_loop(Lane *ln) {
  Server *s = ln->srv;
  cudaSetDevice(s->ctx->device);
  for (;;) {
    std::vector<Request> take;
    uint64_t take_bytes = 0;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_admit.wait(lk, [&] {
        if (s->stop) return true;
        if (ln->waiting.empty()) return false;
        const uint64_t b = ln->waiting.front().bytes;
        return s->admitted_bytes + b <= s->opt.hbm_budget ||
               s->admitted_bytes == 0;
      });
      if (s->stop) {
        // fail everything still waiting in this lane
        for (auto &r : ln->waiting) {
          Result &res = s->results[r.ticket];
          res.done = true;
          res.status = WETRIC_EBUSY;
        }
        ln->waiting.clear();
        s->cv_done.notify_all();
        return;
      }
      // The large lane runs one request at a time through the single-graph
      // path: large graphs gain nothing from sharing a launch.
      const size_t max_take = ln == &s->lanes[1] ? 1 : s->opt.max_batch_graphs;
      uint64_t pairs = 0;
      while (!ln->waiting.empty() && take.size() < max_take) {
        const Request &r = ln->waiting.front();
        if (r.solo && !take.empty()) break;
        const bool fits = s->admitted_bytes + take_bytes + r.bytes <= s->opt.hbm_budget;
        const bool first = take.empty() && s->admitted_bytes == 0;
        if (!fits && !first) break;
        if (!take.empty() && pairs + r.pairs > s->opt.max_batch_pairs) break;
        pairs += r.pairs;
        take_bytes += r.bytes;
        take.push_back(r);
        ln->waiting.pop_front();
        if (take.back().solo) break;
      }
      s->admitted_bytes += take_bytes;
      const Clock::time_point taken = Clock::now();
      for (const Request &r : take)
        s->queue_ms.push_back(
            std::chrono::duration<double, std::milli>(taken - r.arrived).count());
    }
    const uint32_t G = (uint32_t)take.size();
    std::vector<uint64_t> counts(G, 0);
    double prep_ms = 0.0, count_ms = 0.0;
    const int st = G == 1 ? run_single(s, ln, take[0], &counts[0], &prep_ms, &count_ms)
                          : run_batch(s, ln, take, &counts, &prep_ms, &count_ms);
    if (st != WETRIC_OK) {
      cudaStreamSynchronize(ln->stream);
      cudaGetLastError();
    }
    const Clock::time_point now = Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    s->admitted_bytes -= take_bytes;
    s->admit_ms += prep_ms;
    for (const Request &r : take) s->pairs_admitted += r.pairs;
    if (st == WETRIC_EINVAL && G > 1) {
      // One bad request must not fail its batch mates: retry each alone.
      for (auto it = take.rbegin(); it != take.rend(); ++it) {
        it->solo = true;
        ln->waiting.push_front(*it);
      }
      s->cv_admit.notify_all();
      continue;
    }
    s->busy_ms += count_ms;
    ++s->batches;
    s->graphs_in_batches += G;
    for (uint32_t g = 0; g < G; ++g) {
      Result &res = s->results[take[g].ticket];
      res.done = true;
      res.status = st;
      res.count = counts[g];
      res.latency_ms =
          std::chrono::duration<double, std::milli>(now - take[g].arrived).count();
      if (st == WETRIC_OK) {
        ++s->completed;
        s->latencies.push_back(res.latency_ms);
        s->lane_latencies[ln == &s->lanes[1] ? 1 : 0].push_back(res.latency_ms);
      } else {
        ++s->failed;
      }
    }
    s->cv_done.notify_all();
    s->cv_admit.notify_all();
  }
}

double percentile(std::vector<double> v, double p) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = p / 100.0 * (double)(v.size() - 1);
  const size_t lo = (size_t)pos;
  const size_t hi = std::min(lo + 1, v.size() - 1);
  return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}

}  // namespace

}  // namespace wetric

using namespace wetric;

struct wetric_server_s {
  Server s;
};

extern "C" {

void wetric_server_opts_init(wetric_server_opts *o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->hbm_budget = 150ull << 30;
  o->max_batch_graphs = 4096;
  o->spread = 5;
  o->bitmap_len = 8192;
  o->queue_capacity = 1u << 16;
  o->max_batch_pairs = 1ull << 30;
  o->large_pairs = 8ull << 20;
  o->reserve_bytes = 8ull << 30;
}

int wetric_server_create(int device, const wetric_server_opts *opts,
                         wetric_server *out) {
  if (!out) {
    set_error(WETRIC_EINVAL, "NULL argument");
    return WETRIC_EINVAL;
  }
  *out = nullptr;
  wetric_server_opts o;
  if (opts) o = *opts; else wetric_server_opts_init(&o);
  if (!o.hbm_budget) o.hbm_budget = 150ull << 30;
  if (!o.max_batch_graphs) o.max_batch_graphs = 4096;
  if (!o.queue_capacity) o.queue_capacity = 1u << 16;
  if (!o.max_batch_pairs) o.max_batch_pairs = 1ull << 30;
  if (o.bitmap_len % 32 != 0) {
    set_error(WETRIC_EINVAL, "bitmap length is not a multiple of 32");
    return WETRIC_EINVAL;
  }
  DeviceContext *ctx = nullptr;
  int st = get_context(device, &ctx);
  if (st != WETRIC_OK) return st;
  auto *h = new wetric_server_s();
  h->s.ctx = ctx;
  h->s.opt = o;
  // The small lane's stream has the device's highest priority, so its
  // blocks are scheduled ahead of the large lane's as SMs free up.
  int prio_low = 0, prio_high = 0;
  cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  for (int li = 0; li < 2; ++li) {
    Lane &ln = h->s.lanes[li];
    ln.srv = &h->s;
    if (cudaStreamCreateWithPriority(&ln.stream, cudaStreamNonBlocking,
                                     li == 0 ? prio_high : prio_low) != cudaSuccess) {
      cudaGetLastError();
      for (Lane &l2 : h->s.lanes)
        if (l2.stream) cudaStreamDestroy(l2.stream);
      delete h;
      set_error(WETRIC_ECUDA, "stream creation failed");
      return WETRIC_ECUDA;
    }
  }
  // Warm-up before the first request: every lane runs a tiny graph through
  // both paths (loads the kernels, sets up the streams) and grows the memory
  // pool by reserve_bytes once, so no request pays for either.
  for (Lane &ln : h->s.lanes) {
    const int wst = warm_up_lane(&h->s, &ln);
    if (wst != WETRIC_OK) {
      for (Lane &l2 : h->s.lanes) cudaStreamDestroy(l2.stream);
      delete h;
      return wst;
    }
  }
  for (Lane &ln : h->s.lanes) ln.worker = std::thread(lane_loop, &ln);
  *out = h;
  clear_error();
  return WETRIC_OK;
}

int wetric_server_submit(wetric_server h, const uint32_t *src,
                         const uint32_t *dst, uint64_t pairs, uint64_t n,
                         uint32_t flags, uint64_t *ticket) {
  if (!h || !ticket || (pairs && (!src || !dst)) || n == 0) {
    set_error(WETRIC_EINVAL, "bad server request");
    return WETRIC_EINVAL;
  }
  Server &s = h->s;
  Request r;
  r.src = src;
  r.dst = dst;
  r.pairs = pairs;
  r.n = n;
  r.on_device = (flags & WETRIC_CSR_DEVICE) != 0;
  r.arrived = Clock::now();
  r.bytes = estimate_bytes(pairs, n);
  std::lock_guard<std::mutex> lk(s.mu);
  if (s.stop) {
    set_error(WETRIC_EBUSY, "server is stopping");
    return WETRIC_EBUSY;
  }
  if (s.waiting_total() >= s.opt.queue_capacity) {
    set_error(WETRIC_EBUSY, "server queue full");
    return WETRIC_EBUSY;
  }
  r.ticket = s.next_ticket++;
  s.results[r.ticket] = Result();
  const bool large = s.opt.large_pairs && pairs >= s.opt.large_pairs;
  s.lanes[large ? 1 : 0].waiting.push_back(r);
  *ticket = r.ticket;
  s.cv_admit.notify_all();
  return WETRIC_OK;
}

static int take_result(Server &s, uint64_t ticket, uint64_t *count,
                       double *latency_ms) {
  auto it = s.results.find(ticket);
  if (it == s.results.end()) {
    set_error(WETRIC_EINVAL, "unknown ticket %llu", (unsigned long long)ticket);
    return WETRIC_EINVAL;
  }
  if (!it->second.done) return WETRIC_EBUSY;
  const Result r = it->second;
  s.results.erase(it);
  if (r.status != WETRIC_OK) {
    set_error(r.status, "request failed");
    return r.status;
  }
  if (count) *count = r.count;
  if (latency_ms) *latency_ms = r.latency_ms;
  return WETRIC_OK;
}

int wetric_server_poll(wetric_server h, uint64_t ticket, uint64_t *count,
                       double *latency_ms) {
  if (!h) return WETRIC_EINVAL;
  std::lock_guard<std::mutex> lk(h->s.mu);
  return take_result(h->s, ticket, count, latency_ms);
}

int wetric_server_wait(wetric_server h, uint64_t ticket, uint32_t timeout_ms,
                       uint64_t *count, double *latency_ms) {
  if (!h) return WETRIC_EINVAL;
  Server &s = h->s;
  std::unique_lock<std::mutex> lk(s.mu);
  const bool ok = s.cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] {
    auto it = s.results.find(ticket);
    return it == s.results.end() || it->second.done;
  });
  if (!ok) {
    set_error(WETRIC_ETIMEDOUT, "ticket %llu not done after %u ms",
              (unsigned long long)ticket, timeout_ms);
    return WETRIC_ETIMEDOUT;
  }
  return take_result(s, ticket, count, latency_ms);
}

int wetric_server_get_stats(wetric_server h, wetric_server_stats *out) {
  if (!h || !out) return WETRIC_EINVAL;
  Server &s = h->s;
  std::lock_guard<std::mutex> lk(s.mu);
  memset(out, 0, sizeof(*out));
  out->completed = s.completed;
  out->failed = s.failed;
  out->batches = s.batches;
  out->waiting = s.waiting_total();
  out->admitted_bytes = s.admitted_bytes;
  out->mean_batch_graphs = s.batches ? (double)s.graphs_in_batches / (double)s.batches : 0.0;
  out->p50_ms = percentile(s.latencies, 50.0);
  out->p99_ms = percentile(s.latencies, 99.0);
  out->count_busy_ms = s.busy_ms;
  out->admit_busy_ms = s.admit_ms;
  out->pairs_admitted = s.pairs_admitted;
  out->queue_p50_ms = percentile(s.queue_ms, 50.0);
  out->small_p50_ms = percentile(s.lane_latencies[0], 50.0);
  out->small_p99_ms = percentile(s.lane_latencies[0], 99.0);
  out->large_p50_ms = percentile(s.lane_latencies[1], 50.0);
  out->large_p99_ms = percentile(s.lane_latencies[1], 99.0);
  out->large_completed = s.lane_latencies[1].size();
  return WETRIC_OK;
}

void wetric_server_destroy(wetric_server h) {
  if (!h) return;
  Server &s = h->s;
  {
    std::lock_guard<std::mutex> lk(s.mu);
    s.stop = true;
  }
  s.cv_admit.notify_all();
  for (Lane &ln : s.lanes)
    if (ln.worker.joinable()) ln.worker.join();
  cudaSetDevice(s.ctx->device);
  for (Lane &ln : s.lanes) {
    cudaStreamSynchronize(ln.stream);
    cudaStreamDestroy(ln.stream);
  }
  delete h;
}

}  // extern "C"
