// server.cu -- a counting service: requests (one graph each) arrive at any
// time, are admitted against an HBM budget, preprocessed and counted in
// batches while earlier batches are still on the device.
//
// The reference has no serving layer (one graph per process run,
// tc.cu:816-918). Two host threads drive two CUDA streams:
//   * the admit thread takes waiting requests in arrival order while their
//     estimated device footprint fits the budget, folds all of them into
//     one batch (batch_create: one preprocessing pipeline over the disjoint
//     union, resident oriented CSRs), and hands the batch on;
//   * the count thread runs each ready batch's persistent count
//     (batch_count, CUDA-graph replay off) on its own stream, completes the
//     batch's tickets and releases its memory.
// So a request that arrives while a batch is counting is preprocessed on
// the other stream at the same time, and joins the next launch as soon as
// memory allows: continuous batching rather than a FIFO of single runs.
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

struct ReadyBatch {
  std::unique_ptr<Batch> batch;
  std::vector<Request> reqs;
  uint64_t bytes = 0;
};

}  // namespace

struct Server {
  DeviceContext *ctx = nullptr;
  cudaStream_t admit_stream = nullptr, count_stream = nullptr;
  wetric_server_opts opt{};
  std::mutex mu;
  std::condition_variable cv_admit, cv_count, cv_done;
  std::deque<Request> waiting;
  std::deque<ReadyBatch> ready;
  std::unordered_map<uint64_t, Result> results;
  uint64_t next_ticket = 1;
  uint64_t admitted_bytes = 0;
  bool stop = false;        // admission stops
  bool stop_count = false;  // counting stops once `ready` drains
  std::thread admit_thread, count_thread;
  // statistics
  uint64_t completed = 0, batches = 0, failed = 0, graphs_in_batches = 0;
  std::vector<double> latencies;
  double busy_ms = 0.0;
  double admit_ms = 0.0;
  uint64_t pairs_admitted = 0;
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

void admit_loop(Server *s) {
  cudaSetDevice(s->ctx->device);
  for (;;) {
    std::vector<Request> take;
    uint64_t take_bytes = 0;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_admit.wait(lk, [&] {
        if (s->stop) return true;
        if (s->waiting.empty()) return false;
        const uint64_t b = s->waiting.front().bytes;
        return s->admitted_bytes + b <= s->opt.hbm_budget ||
               s->admitted_bytes == 0;
      });
      if (s->stop && s->waiting.empty()) return;
      if (s->stop) {
        // fail everything still waiting
        for (auto &r : s->waiting) {
          Result &res = s->results[r.ticket];
          res.done = true;
          res.status = WETRIC_EBUSY;
        }
        s->waiting.clear();
        s->cv_done.notify_all();
        return;
      }
      uint64_t pairs = 0;
      while (!s->waiting.empty() && take.size() < s->opt.max_batch_graphs) {
        const Request &r = s->waiting.front();
        if (r.solo && !take.empty()) break;
        const bool fits = s->admitted_bytes + take_bytes + r.bytes <= s->opt.hbm_budget;
        const bool first = take.empty() && s->admitted_bytes == 0;
        if (!fits && !first) break;
        if (!take.empty() && pairs + r.pairs > s->opt.max_batch_pairs) break;
        pairs += r.pairs;
        take_bytes += r.bytes;
        take.push_back(r);
        s->waiting.pop_front();
        if (take.back().solo) break;
      }
      s->admitted_bytes += take_bytes;
    }
    // Build the batch: concatenate the requests' pairs on the device.
    const uint32_t G = (uint32_t)take.size();
    std::vector<uint64_t> off(G + 1, 0), n(G);
    for (uint32_t g = 0; g < G; ++g) {
      off[g + 1] = off[g] + take[g].pairs;
      n[g] = take[g].n;
    }
    ReadyBatch rb;
    rb.reqs = std::move(take);
    rb.bytes = take_bytes;
    int st = WETRIC_OK;
    Scratch<uint32_t> us, ud;
    auto build = [&]() -> int {
      WETRIC_TRY(us.alloc(s->ctx, s->admit_stream, off[G]));
      WETRIC_TRY(ud.alloc(s->ctx, s->admit_stream, off[G]));
      for (uint32_t g = 0; g < G; ++g) {
        const Request &r = rb.reqs[g];
        if (!r.pairs) continue;
        const cudaMemcpyKind k =
            r.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        WETRIC_CUDA_TRY(cudaMemcpyAsync(us.ptr + off[g], r.src, r.pairs * 4, k,
                                        s->admit_stream));
        WETRIC_CUDA_TRY(cudaMemcpyAsync(ud.ptr + off[g], r.dst, r.pairs * 4, k,
                                        s->admit_stream));
      }
      BatchOptions bo;
      bo.spread = s->opt.spread ? s->opt.spread : 5;
      bo.bitmap_len = s->opt.bitmap_len;
      bo.use_graph = false;  // each batch is counted once
      rb.batch = std::make_unique<Batch>();
      WETRIC_TRY(batch_create(s->ctx, us.ptr, ud.ptr, off.data(), n.data(), G,
                              true, bo, rb.batch.get(), s->admit_stream));
      us.release();
      ud.release();
      WETRIC_CUDA_TRY(cudaStreamSynchronize(s->admit_stream));
      return WETRIC_OK;
    };
    const Clock::time_point b0 = Clock::now();
    st = build();
    const double build_ms =
        std::chrono::duration<double, std::milli>(Clock::now() - b0).count();
    std::lock_guard<std::mutex> lk(s->mu);
    s->admit_ms += build_ms;
    s->pairs_admitted += off[G];
    if (st != WETRIC_OK && rb.reqs.size() > 1 && st == WETRIC_EINVAL) {
      // One bad request must not fail its batch mates: retry each alone.
      rb.batch.reset();
      s->admitted_bytes -= rb.bytes;
      for (auto it = rb.reqs.rbegin(); it != rb.reqs.rend(); ++it) {
        it->solo = true;
        s->waiting.push_front(*it);
      }
      s->cv_admit.notify_all();
      continue;
    }
    if (st != WETRIC_OK) {
      rb.batch.reset();
      s->admitted_bytes -= rb.bytes;
      for (auto &r : rb.reqs) {
        Result &res = s->results[r.ticket];
        res.done = true;
        res.status = st;
        ++s->failed;
      }
      s->cv_done.notify_all();
      s->cv_admit.notify_all();
      continue;
    }
    s->ready.push_back(std::move(rb));
    s->cv_count.notify_all();
  }
}

void count_loop(Server *s) {
  cudaSetDevice(s->ctx->device);
  for (;;) {
    ReadyBatch rb;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_count.wait(lk, [&] { return s->stop_count || !s->ready.empty(); });
      if (s->ready.empty()) return;  // admission finished and nothing left
      rb = std::move(s->ready.front());
      s->ready.pop_front();
    }
    const uint32_t G = (uint32_t)rb.reqs.size();
    std::vector<uint64_t> counts(G, 0);
    double ms = 0;
    uint32_t launches = 0;
    const int st = batch_count(rb.batch.get(), counts.data(), &ms, &launches,
                               s->count_stream);
    const Clock::time_point now = Clock::now();
    // Release the batch's memory (stream-ordered on the admission stream,
    // where the next batch allocates).
    rb.batch.reset();
    std::lock_guard<std::mutex> lk(s->mu);
    s->admitted_bytes -= rb.bytes;
    s->busy_ms += ms;
    ++s->batches;
    s->graphs_in_batches += G;
    for (uint32_t g = 0; g < G; ++g) {
      Result &res = s->results[rb.reqs[g].ticket];
      res.done = true;
      res.status = st;
      res.count = counts[g];
      res.latency_ms =
          std::chrono::duration<double, std::milli>(now - rb.reqs[g].arrived).count();
      if (st == WETRIC_OK) {
        ++s->completed;
        s->latencies.push_back(res.latency_ms);
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
  if (cudaStreamCreateWithFlags(&h->s.admit_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->s.count_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    if (h->s.admit_stream) cudaStreamDestroy(h->s.admit_stream);
    delete h;
    set_error(WETRIC_ECUDA, "stream creation failed");
    return WETRIC_ECUDA;
  }
  h->s.admit_thread = std::thread(admit_loop, &h->s);
  h->s.count_thread = std::thread(count_loop, &h->s);
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
  if (s.waiting.size() >= s.opt.queue_capacity) {
    set_error(WETRIC_EBUSY, "server queue full");
    return WETRIC_EBUSY;
  }
  r.ticket = s.next_ticket++;
  s.results[r.ticket] = Result();
  s.waiting.push_back(r);
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
  out->waiting = s.waiting.size();
  out->admitted_bytes = s.admitted_bytes;
  out->mean_batch_graphs = s.batches ? (double)s.graphs_in_batches / (double)s.batches : 0.0;
  out->p50_ms = percentile(s.latencies, 50.0);
  out->p99_ms = percentile(s.latencies, 99.0);
  out->count_busy_ms = s.busy_ms;
  out->admit_busy_ms = s.admit_ms;
  out->pairs_admitted = s.pairs_admitted;
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
  if (s.admit_thread.joinable()) s.admit_thread.join();
  {
    std::lock_guard<std::mutex> lk(s.mu);
    s.stop_count = true;
  }
  s.cv_count.notify_all();
  if (s.count_thread.joinable()) s.count_thread.join();
  cudaSetDevice(s.ctx->device);
  cudaStreamSynchronize(s.admit_stream);
  cudaStreamSynchronize(s.count_stream);
  cudaStreamDestroy(s.admit_stream);
  cudaStreamDestroy(s.count_stream);
  delete h;
}

}  // extern "C"
