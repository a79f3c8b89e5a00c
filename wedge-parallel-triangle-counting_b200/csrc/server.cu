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
#include "serve.cuh"

namespace wetric {

namespace {

using Clock = std::chrono::steady_clock;

// Pairs the server made itself from a submitted CSR: kept alive by every
// copy of the request until the last one is dropped (after its
// preprocessing, which has synchronised its stream by then).
struct OwnedPairs {
  std::vector<uint32_t> hsrc, hdst;  // host CSR input
  Scratch<uint32_t> dsrc, ddst;      // device CSR input
};

struct Request {
  uint64_t ticket = 0;
  const uint32_t *src = nullptr, *dst = nullptr;
  uint64_t pairs = 0, n = 0;
  bool on_device = false;
  Clock::time_point arrived;
  uint64_t bytes = 0;  // admission estimate
  bool solo = false;   // re-admitted alone after its batch failed
  std::shared_ptr<OwnedPairs> owned;
};

// Row of every column of a CSR: src[j] = the row holding entry j (the
// last row whose offset is <= j), dst[j] = col_ind[j].
template <typename Off>
__global__ void k_csr_to_pairs(const Off *__restrict__ rp, const uint32_t *__restrict__ ci,
                               uint64_t n, uint64_t m, uint32_t *__restrict__ src,
                               uint32_t *__restrict__ dst) {
  for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < m;
       j += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t lo = 0, len = n;
    while (len > 1) {
      const uint64_t h = len >> 1;
      if ((uint64_t)rp[lo + h] <= j) lo += h;
      len -= h;
    }
    src[j] = (uint32_t)lo;
    dst[j] = ci[j];
  }
}

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
  // resident mode: more workers preprocessing this lane's requests side by
  // side, each on its own stream (preprocessing is a chain of small
  // kernels and read-backs, so one thread alone cannot keep up with many
  // small requests)
  std::vector<std::thread> more;
  std::vector<cudaStream_t> more_streams;
};

// Workers of the small lane in resident mode (the large lane has one).
constexpr int kSmallPrepWorkers = 4;

// A request folded into the resident kernel: its ticket, arrival, lane,
// admission bytes and how many of its tiles are published.
struct Live {
  uint64_t ticket = 0;
  Clock::time_point arrived;
  int lane = 0;
  uint64_t tiles = 0, fed = 0, item = 0;  // item: tiles per queue item
  uint64_t items_left = 0;                // reserved items not yet published
};

struct Server {
  DeviceContext *ctx = nullptr;
  wetric_server_opts opt{};
  std::mutex mu;
  std::condition_variable cv_admit, cv_done, cv_space, cv_monitor;
  // resident mode
  ServeEngine *eng = nullptr;
  std::thread monitor;
  std::unordered_map<uint32_t, Live> live;  // slot -> request
  std::deque<uint32_t> feeding;             // slots with unpublished tiles
  bool draining = false;                    // no new slots until recycled
  uint64_t items_reserved = 0;              // items live requests will still publish
  uint64_t freed_seen = 0, recycles = 0;
  int lanes_running = 0;
  uint32_t lane_phase[2] = {0, 0};  // see wetric_server_stats::lane_phase
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

// ------------------------------------------------------ resident mode

// Queue items of fed (large) requests kept ahead of the kernel at once.
constexpr uint64_t kFeedDepth = 4;

// Items a request of `tiles` tiles is fed in: item_tiles each, at most
// kMaxItemsPerRequest (larger requests get larger items).
constexpr uint64_t kMaxItemsPerRequest = 64;
uint64_t item_size(const Server *s, uint64_t tiles) {
  const uint64_t floor_size = ceil_div(tiles, kMaxItemsPerRequest);
  return s->opt.item_tiles > floor_size ? s->opt.item_tiles : floor_size;
}

// Copies the request's pairs (host input), orients them into plan->csr and
// builds every structure of its count on the lane's stream.
int prep_resident(Server *s, cudaStream_t st, const Request &r, ServePlan *plan) {
  Scratch<uint32_t> us, ud;
  const uint32_t *src = r.src, *dst = r.dst;
  if (!r.on_device && r.pairs) {
    WETRIC_TRY(us.alloc(s->ctx, st, r.pairs));
    WETRIC_TRY(ud.alloc(s->ctx, st, r.pairs));
    WETRIC_CUDA_TRY(cudaMemcpyAsync(us.ptr, r.src, r.pairs * 4, cudaMemcpyHostToDevice, st));
    WETRIC_CUDA_TRY(cudaMemcpyAsync(ud.ptr, r.dst, r.pairs * 4, cudaMemcpyHostToDevice, st));
    src = us.ptr;
    dst = ud.ptr;
  }
  WETRIC_TRY(orient_pairs(s->ctx, st, src, dst, r.pairs, r.n, &plan->csr));
  us.release();
  ud.release();
  return serve_prepare(s->ctx, st, s->opt.spread ? s->opt.spread : 5, s->opt.bitmap_len, plan);
}

void finish_request(Server *s, uint64_t ticket, int status, uint64_t count,
                    Clock::time_point arrived, int lane) {
  Result &res = s->results[ticket];
  res.done = true;
  res.status = status;
  res.count = count;
  res.latency_ms = std::chrono::duration<double, std::milli>(Clock::now() - arrived).count();
  if (status == WETRIC_OK) {
    ++s->completed;
    s->latencies.push_back(res.latency_ms);
    s->lane_latencies[lane].push_back(res.latency_ms);
  } else {
    ++s->failed;
  }
}

void lane_loop_resident(Lane *ln, cudaStream_t wst) {
  Server *s = ln->srv;
  cudaSetDevice(s->ctx->device);
  const int li = ln == &s->lanes[1] ? 1 : 0;
  for (;;) {
    Request r;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->lane_phase[li] = 0;
      s->cv_admit.wait(lk, [&] {
        if (s->stop) return true;
        if (ln->waiting.empty()) return false;
        return s->admitted_bytes + ln->waiting.front().bytes <= s->opt.hbm_budget ||
               s->admitted_bytes == 0;
      });
      if (s->stop) {
        for (auto &w : ln->waiting) {
          Result &res = s->results[w.ticket];
          res.done = true;
          res.status = WETRIC_EBUSY;
        }
        ln->waiting.clear();
        --s->lanes_running;
        s->cv_done.notify_all();
        s->cv_monitor.notify_all();
        return;
      }
      r = ln->waiting.front();
      ln->waiting.pop_front();
      s->admitted_bytes += r.bytes;
      s->lane_phase[li] = 1;
      s->queue_ms.push_back(
          std::chrono::duration<double, std::milli>(Clock::now() - r.arrived).count());
    }
    const Clock::time_point t0 = Clock::now();
    std::unique_ptr<ServePlan> plan(new ServePlan());
    int st = prep_resident(s, wst, r, plan.get());
    plan->bytes = r.bytes;
    const uint64_t tiles = plan->tiles;
    std::unique_lock<std::mutex> lk(s->mu);
    s->admit_ms += std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
    s->pairs_admitted += r.pairs;
    if (st != WETRIC_OK) {
      lk.unlock();
      cudaStreamSynchronize(wst);
      cudaGetLastError();
      plan.reset();
      lk.lock();
      s->admitted_bytes -= r.bytes;
      finish_request(s, r.ticket, st, 0, r.arrived, li);
      s->cv_done.notify_all();
      s->cv_admit.notify_all();
      continue;
    }
    // Register and publish (wait while the engine drains for a recycle).
    // The request's queue items are reserved now, so the sequence space
    // cannot run out in the middle of feeding it.
    const uint64_t item = item_size(s, tiles);
    const uint64_t need = tiles ? ceil_div(tiles, item) : 0;
    uint32_t slot = 0;
    s->lane_phase[li] = 2;
    for (;;) {
      if (s->stop) {
        st = WETRIC_EBUSY;  // the server is closing: drop the request
        break;
      }
      if (!s->draining) {
        uint32_t slots_left = 0, items_left = 0;
        serve_space_left(s->eng, &slots_left, &items_left);
        if (slots_left >= 1 && s->items_reserved + need <= items_left) {
          st = serve_add(s->eng, plan, &slot);
          if (st != WETRIC_EBUSY) break;
        }
        s->draining = true;  // sequence space used up: recycle first
        s->cv_monitor.notify_all();
      }
      s->cv_space.wait(lk);
    }
    s->lane_phase[li] = 3;
    if (st != WETRIC_OK) {
      lk.unlock();
      plan.reset();  // frees its memory in its stream's order
      lk.lock();
      s->admitted_bytes -= r.bytes;
      finish_request(s, r.ticket, st, 0, r.arrived, li);
      s->cv_done.notify_all();
      continue;
    }
    Live l;
    l.ticket = r.ticket;
    l.arrived = r.arrived;
    l.lane = li;
    l.tiles = tiles;
    l.item = item;
    l.items_left = need;
    s->items_reserved += need;
    const uint64_t first = tiles < item ? tiles : item;
    if (first) {
      st = serve_publish(s->eng, slot, 0, first);
      --l.items_left;
      --s->items_reserved;
    }
    l.fed = first;
    s->live[slot] = l;
    if (st == WETRIC_OK && first < tiles) s->feeding.push_back(slot);
    s->cv_monitor.notify_all();
    s->lane_phase[li] = 0;
    lk.unlock();
    serve_kick(s->eng);
  }
}

void monitor_loop(Server *s) {
  cudaSetDevice(s->ctx->device);
  std::vector<std::pair<uint32_t, uint64_t>> done;
  const uint64_t recycle_bytes =
      std::min<uint64_t>(s->opt.hbm_budget / 4, 32ull << 30);
  // On close, requests still registered get kStopDrainSeconds to complete;
  // after that they fail (EBUSY) and the engine is stopped regardless.
  constexpr int kStopDrainSeconds = 10;
  Clock::time_point stop_seen{};
  bool stop_noted = false;
  for (;;) {
    serve_poll(s->eng, &done);
    const uint64_t freed = serve_freed_bytes(s->eng);
    uint64_t taken = 0, published = 0;
    serve_queue_state(s->eng, &taken, &published);
    bool recycle = false;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      for (const auto &d : done) {
        auto it = s->live.find(d.first);
        if (it == s->live.end()) continue;
        finish_request(s, it->second.ticket, WETRIC_OK, d.second, it->second.arrived,
                       it->second.lane);
        s->live.erase(it);
      }
      if (!done.empty()) s->cv_done.notify_all();
      if (freed > s->freed_seen) {
        s->admitted_bytes -= std::min(s->admitted_bytes, freed - s->freed_seen);
        s->freed_seen = freed;
        s->cv_admit.notify_all();
      }
      // Feed large requests an item at a time, round robin, keeping only a
      // few items ahead of the kernel so newly published small requests
      // are taken soon.
      while (!s->feeding.empty() && published - taken < kFeedDepth) {
        const uint32_t slot = s->feeding.front();
        s->feeding.pop_front();
        Live &l = s->live[slot];
        const uint64_t t1 = std::min(l.tiles, l.fed + l.item);
        if (serve_publish(s->eng, slot, l.fed, t1) != WETRIC_OK) {
          s->feeding.push_front(slot);  // cannot happen: the items are reserved
          break;
        }
        ++published;
        if (l.items_left) {
          --l.items_left;
          --s->items_reserved;
        }
        l.fed = t1;
        if (t1 < l.tiles) s->feeding.push_back(slot);
      }
      uint32_t slots_left = 0, items_left = 0;
      serve_space_left(s->eng, &slots_left, &items_left);
      if (serve_retired_bytes(s->eng) > recycle_bytes || slots_left < 2 ||
          items_left < s->items_reserved + kMaxItemsPerRequest)
        s->draining = true;
      recycle = s->draining && s->live.empty();
      if (s->stop && s->lanes_running == 0) {
        if (!stop_noted) {
          stop_noted = true;
          stop_seen = Clock::now();
        }
        if (s->live.empty()) return;
        if (Clock::now() - stop_seen > std::chrono::seconds(kStopDrainSeconds)) {
          for (const auto &kv : s->live)
            finish_request(s, kv.second.ticket, WETRIC_EBUSY, 0, kv.second.arrived,
                           kv.second.lane);
          s->live.clear();
          s->feeding.clear();
          s->cv_done.notify_all();
          return;
        }
      }
    }
    if (recycle) {
      serve_recycle(s->eng);
      std::lock_guard<std::mutex> lk(s->mu);
      s->draining = false;
      ++s->recycles;
      s->cv_space.notify_all();
    }
    serve_kick(s->eng);
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_monitor.wait_for(lk, std::chrono::microseconds(50));
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
  o->resident = 0;
  o->item_tiles = 65536;
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
  if (!o.item_tiles) o.item_tiles = 65536;
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
  if (o.resident) {
    ServeEngineOptions eo;
    const int est = serve_engine_create(ctx, eo, &h->s.eng);
    if (est != WETRIC_OK) {
      for (Lane &l2 : h->s.lanes) cudaStreamDestroy(l2.stream);
      delete h;
      return est;
    }
    // load the resident kernel once (a launch that idles out at once)
    uint32_t code = 0;
    double ms = 0;
    const int pst = serve_idle_probe(ctx, 10, &code, &ms);
    if (pst != WETRIC_OK) {
      serve_engine_destroy(h->s.eng);
      for (Lane &l2 : h->s.lanes) cudaStreamDestroy(l2.stream);
      delete h;
      return pst;
    }
    int workers = 0;
    for (int li = 0; li < 2; ++li) {
      Lane &ln = h->s.lanes[li];
      int prio = 0;
      cudaStreamGetPriority(ln.stream, &prio);
      for (int k = 1; li == 0 && k < kSmallPrepWorkers; ++k) {
        cudaStream_t x = nullptr;
        if (cudaStreamCreateWithPriority(&x, cudaStreamNonBlocking, prio) != cudaSuccess) {
          cudaGetLastError();
          break;
        }
        ln.more_streams.push_back(x);
      }
      workers += 1 + (int)ln.more_streams.size();
    }
    h->s.lanes_running = workers;
    for (Lane &ln : h->s.lanes) {
      ln.worker = std::thread(lane_loop_resident, &ln, ln.stream);
      for (cudaStream_t x : ln.more_streams) ln.more.emplace_back(lane_loop_resident, &ln, x);
    }
    h->s.monitor = std::thread(monitor_loop, &h->s);
  } else {
    for (Lane &ln : h->s.lanes) ln.worker = std::thread(lane_loop, &ln);
  }
  *out = h;
  clear_error();
  return WETRIC_OK;
}

static int enqueue_request(Server &s, Request &r, uint64_t *ticket) {
  r.arrived = Clock::now();
  r.bytes = estimate_bytes(r.pairs, r.n);
  const uint64_t pairs = r.pairs;
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

int wetric_server_submit(wetric_server h, const uint32_t *src,
                         const uint32_t *dst, uint64_t pairs, uint64_t n,
                         uint32_t flags, uint64_t *ticket) {
  if (!h || !ticket || (pairs && (!src || !dst)) || n == 0) {
    set_error(WETRIC_EINVAL, "bad server request");
    return WETRIC_EINVAL;
  }
  Request r;
  r.src = src;
  r.dst = dst;
  r.pairs = pairs;
  r.n = n;
  r.on_device = (flags & WETRIC_CSR_DEVICE) != 0;
  return enqueue_request(h->s, r, ticket);
}

int wetric_server_submit_csr(wetric_server h, const wetric_csr *csr, uint64_t *ticket) {
  if (!h || !ticket || !csr || csr->n == 0 || !csr->row_ptr ||
      csr->n > (1ull << 32)) {
    set_error(WETRIC_EINVAL, "bad server request");
    return WETRIC_EINVAL;
  }
  Server &s = h->s;
  const bool dev = (csr->flags & WETRIC_CSR_DEVICE) != 0;
  const bool off32 = (csr->flags & WETRIC_CSR_OFFSETS32) != 0;
  const uint64_t n = csr->n;
  auto owned = std::make_shared<OwnedPairs>();
  uint64_t m = 0;
  if (!dev) {
    m = off32 ? static_cast<const uint32_t *>(csr->row_ptr)[n]
              : static_cast<const uint64_t *>(csr->row_ptr)[n];
    if (m && !csr->col_ind) {
      set_error(WETRIC_EINVAL, "bad server request");
      return WETRIC_EINVAL;
    }
    owned->hsrc.resize(m);
    owned->hdst.resize(m);
    const int64_t rows = (int64_t)n;
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t v = 0; v < rows; ++v) {
      const uint64_t b = off32 ? static_cast<const uint32_t *>(csr->row_ptr)[v]
                               : static_cast<const uint64_t *>(csr->row_ptr)[v];
      const uint64_t e = off32 ? static_cast<const uint32_t *>(csr->row_ptr)[v + 1]
                               : static_cast<const uint64_t *>(csr->row_ptr)[v + 1];
      for (uint64_t j = b; j < e && j < m; ++j) {
        owned->hsrc[j] = (uint32_t)v;
        owned->hdst[j] = csr->col_ind[j];
      }
    }
  } else {
    // expand on the device (the library's stream), then wait for it, so
    // the lanes read finished pairs
    WETRIC_CUDA_TRY(cudaSetDevice(s.ctx->device));
    const cudaStream_t st = s.ctx->stream;
    if (off32) {
      uint32_t m32 = 0;
      WETRIC_CUDA_TRY(cudaMemcpy(&m32, static_cast<const uint32_t *>(csr->row_ptr) + n, 4,
                                 cudaMemcpyDeviceToHost));
      m = m32;
    } else {
      WETRIC_CUDA_TRY(cudaMemcpy(&m, static_cast<const uint64_t *>(csr->row_ptr) + n, 8,
                                 cudaMemcpyDeviceToHost));
    }
    if (m && !csr->col_ind) {
      set_error(WETRIC_EINVAL, "bad server request");
      return WETRIC_EINVAL;
    }
    WETRIC_TRY(owned->dsrc.alloc(s.ctx, st, m));
    WETRIC_TRY(owned->ddst.alloc(s.ctx, st, m));
    if (m) {
      const uint64_t cap = (uint64_t)s.ctx->sm_count * 32;
      uint64_t grid = ceil_div(m, 256);
      if (grid > cap) grid = cap;
      if (off32)
        k_csr_to_pairs<uint32_t><<<(unsigned)grid, 256, 0, st>>>(
            static_cast<const uint32_t *>(csr->row_ptr), csr->col_ind, n, m,
            owned->dsrc.ptr, owned->ddst.ptr);
      else
        k_csr_to_pairs<uint64_t><<<(unsigned)grid, 256, 0, st>>>(
            static_cast<const uint64_t *>(csr->row_ptr), csr->col_ind, n, m,
            owned->dsrc.ptr, owned->ddst.ptr);
      WETRIC_LAUNCH_CHECK();
    }
    WETRIC_CUDA_TRY(cudaStreamSynchronize(st));
  }
  Request r;
  r.src = dev ? owned->dsrc.ptr : owned->hsrc.data();
  r.dst = dev ? owned->ddst.ptr : owned->hdst.data();
  r.pairs = m;
  r.n = n;
  r.on_device = dev;
  r.owned = std::move(owned);
  return enqueue_request(s, r, ticket);
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
  out->recycles = s.recycles;
  if (s.eng) {
    serve_launch_info(s.eng, &out->resident_launches, &out->resident_last_exit);
    serve_queue_state(s.eng, &out->items_taken, &out->items_published);
    out->launch_errors = (uint32_t)serve_launch_errors(s.eng, &out->launch_error_code);
  }
  out->live = s.live.size();
  out->feeding = s.feeding.size();
  out->draining = s.draining ? 1u : 0u;
  out->lane_phase[0] = s.lane_phase[0];
  out->lane_phase[1] = s.lane_phase[1];
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
  s.cv_space.notify_all();
  for (Lane &ln : s.lanes) {
    if (ln.worker.joinable()) ln.worker.join();
    for (std::thread &t : ln.more)
      if (t.joinable()) t.join();
  }
  s.cv_monitor.notify_all();
  if (s.monitor.joinable()) s.monitor.join();
  cudaSetDevice(s.ctx->device);
  if (s.eng) serve_engine_destroy(s.eng);
  for (Lane &ln : s.lanes) {
    cudaStreamSynchronize(ln.stream);
    cudaStreamDestroy(ln.stream);
    for (cudaStream_t x : ln.more_streams) {
      cudaStreamSynchronize(x);
      cudaStreamDestroy(x);
    }
  }
  delete h;
}

}  // extern "C"
