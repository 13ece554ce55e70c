// serve.cpp - request loop with device-wide HBM-budget admission, size lanes
// and continuous batching (the C ABI's fpx_serve_*).  The reference has no server; this serves its
// batch/serve workload (mixed operations, sizes and moduli arriving over time)
// with the same per-request results as the single-operation functions.
#include <algorithm>
#include <atomic>
#include <bit>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"
#include "fpx_b200.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t ticket;
  fpx_job* job;
  size_t bytes;
  Clock::time_point t_submit, t_done;
  bool done = false;
};

bool native_size(uint32_t p, int logN) {
  return (p & 1u) && p < (1u << 30) && logN >= 1 && logN <= 25 && logN <= fpx::v2_of(p);
}

size_t pow2_at_least(size_t x) { return x <= 1 ? 1 : size_t(1) << std::bit_width(x - 1); }

}  // namespace

// Planned device bytes of one request: operands and results, plus the
// transform scratch its products take at their largest stage (two N-word
// buffers per product, three auxiliary primes when the modulus is not an NTT
// prime for that size), plus the Newton loops' persistent buffers.
extern "C" size_t fpx_serve_plan_bytes(const fpx_job* j) {
  if (!j || j->p < 2) return 0;
  const uint32_t p = j->p;
  const size_t B = size_t(1) << 23;  // CRT block (crt_convolution.hpp:19)
  auto prod2 = [&](size_t la, size_t lb) -> size_t {  // scratch words of one la x lb product
    const size_t full = la + lb - 1;
    const size_t N = pow2_at_least(full);
    const int logN = std::countr_zero(N);
    if (native_size(p, logN)) return 2 * N;
    if (la > B || lb > B)  // blocked: every block's spectrum at 2^24 points, two work buffers, three residue arrays
      return ((la + B - 1) / B + (lb + B - 1) / B + 2) * (2 * B) + 3 * full;
    return 3 * (2 * N + full);
  };
  auto prod = [&](size_t full) -> size_t { return prod2(full / 2 + 1, full / 2 + 1); };
  size_t in = 0, out = 0, scratch = 0;
  switch (j->op) {
    case FPX_OP_CONV: {
      const size_t la = std::min(j->la, j->n), lb = std::min(j->lb, j->n);
      if (!la || !lb) return 64;
      in = la + lb;
      out = std::min(la + lb - 1, j->n);
      scratch = prod2(la, lb);
      break;
    }
    case FPX_OP_INV:
    case FPX_OP_LOG:
    case FPX_OP_EXP:
    case FPX_OP_SQRT:
    case FPX_OP_POW: {
      const size_t n = j->n;
      in = j->op == FPX_OP_POW ? j->la : std::min(j->la, n);
      out = n;
      const size_t per_step = prod(2 * n);
      const size_t persistent = j->op == FPX_OP_EXP ? 9 * n : (j->op == FPX_OP_INV ? 3 * n : 6 * n);
      scratch = persistent + per_step;
      if (j->op == FPX_OP_POW) scratch += 3 * n;
      break;
    }
    case FPX_OP_DIVMOD: {
      in = j->la + j->lb;
      out = j->la + j->lb;
      scratch = 4 * j->la + prod(2 * j->la);
      break;
    }
    default:
      return 0;
  }
  return 4 * (in + out + scratch) + 1024;
}

// Size lanes: requests of at most 2^kSmallLaneLog terms (the longest operand,
// or the series length) go to the small lane, the rest to the large lane.  Each
// lane has its own queue and workers, so a short request is never batched with
// (and held behind) a 2^22-term one.
constexpr int kSmallLaneLog = 17;

int lane_of(const fpx_job* j) {
  size_t n = 0;
  switch (j->op) {
    case FPX_OP_CONV: n = std::max(std::min(j->la, j->n), std::min(j->lb, j->n)); break;
    case FPX_OP_DIVMOD: n = std::max(j->la, j->lb); break;
    default: n = j->n;
  }
  return n <= (size_t(1) << kSmallLaneLog) ? 0 : 1;
}

struct fpx_server {
  int device = 0;
  fpx_serve_config cfg{};
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> queue[2];  // per lane, arrival order
  std::unordered_map<uint64_t, std::unique_ptr<Request>> all;
  uint64_t next_ticket = 1;
  bool stopping = false;
  std::vector<std::thread> workers;
  std::vector<std::unique_ptr<fpx::Engine>> engines;
  fpx_serve_stats stats{};
  int small_workers = 1;
  // Device-wide admission: planned bytes of every micro-batch on the GPU,
  // charged when it is formed and refunded when it completes.
  size_t in_flight = 0;
  // The large lane's oldest request does not fit the bytes left: no lane admits
  // new work until it does, so large requests cannot be starved by small ones.
  bool large_waiting = false;

  bool drained() const { return queue[0].empty() && queue[1].empty(); }

  // Forms one micro-batch for a worker of `lane` (mu held): from the lane's own
  // queue, or, for the large lane with nothing of its own, from the small lane.
  // Returns the planned bytes taken (mine empty: nothing admissible now).
  size_t admit(int lane, std::vector<Request*>& mine) {
    const bool own = !queue[lane].empty();
    if (!own && lane == 0) return 0;
    std::deque<Request*>& q = own ? queue[lane] : queue[0];
    if (large_waiting && !(own && lane == 1)) return 0;
    // One micro-batch takes at most its lane's share of the budget (the budget
    // over the lane's workers), so that a backlog does not turn into one
    // budget-sized micro-batch that every other request waits behind; a
    // single request above the share still goes, alone.
    const int lane_workers = lane == 0 ? small_workers : (int)engines.size() - small_workers;
    const size_t share = cfg.hbm_budget_bytes / (size_t)std::max(1, lane_workers);
    size_t bytes = 0;
    while (!q.empty() && mine.size() < cfg.max_batch_jobs) {
      Request* r = q.front();
      const size_t total = in_flight + bytes + r->bytes;
      const bool alone = in_flight == 0 && mine.empty();  // a request larger than the budget runs alone
      if (total > cfg.hbm_budget_bytes && !alone) {
        if (own && lane == 1 && mine.empty()) large_waiting = true;
        break;
      }
      if (!mine.empty() && bytes + r->bytes > share) break;
      if (r->bytes > cfg.hbm_budget_bytes) ++stats.oversize_requests;
      bytes += r->bytes;
      mine.push_back(r);
      q.pop_front();
    }
    if (!mine.empty() && own && lane == 1) large_waiting = false;
    return bytes;
  }

  void worker(int w) {
    fpx::Engine& eng = *engines[w];
    const int lane = w < small_workers ? 0 : 1;
    cudaSetDevice(device);
    std::vector<Request*> mine;
    std::vector<fpx_job> jobs;
    for (;;) {
      mine.clear();
      size_t bytes = 0;
      {
        std::unique_lock<std::mutex> g(mu);
        for (;;) {
          bytes = admit(lane, mine);
          if (!mine.empty()) break;
          if (stopping && drained()) return;
          cv_work.wait(g);
        }
        in_flight += bytes;
        ++stats.batches;
        stats.max_batch_jobs_seen = std::max<uint64_t>(stats.max_batch_jobs_seen, mine.size());
        stats.max_batch_bytes_seen = std::max<uint64_t>(stats.max_batch_bytes_seen, bytes);
        stats.max_in_flight_bytes = std::max<uint64_t>(stats.max_in_flight_bytes, in_flight);
      }
      cv_work.notify_all();  // another worker may admit from what is left
      jobs.resize(mine.size());
      for (size_t i = 0; i < mine.size(); ++i) jobs[i] = *mine[i]->job;
      int whole = FPX_OK;
      try {
        eng.check(cudaSetDevice(device), "cudaSetDevice");
        eng.batch_host(jobs.data(), jobs.size(), cfg.repr);
      } catch (const fpx::Error& e) {
        whole = e.code;
      } catch (...) {
        whole = FPX_EINVAL;
      }
      const Clock::time_point now = Clock::now();
      {
        std::lock_guard<std::mutex> g(mu);
        for (size_t i = 0; i < mine.size(); ++i) {
          fpx_job* dst = mine[i]->job;
          dst->status = whole != FPX_OK ? whole : jobs[i].status;
          dst->out_len = whole != FPX_OK ? 0 : jobs[i].out_len;
          dst->out2_len = whole != FPX_OK ? 0 : jobs[i].out2_len;
          mine[i]->t_done = now;
          mine[i]->done = true;
          ++stats.completed;
        }
        in_flight -= bytes;
      }
      cv_done.notify_all();
      cv_work.notify_all();  // bytes were refunded
    }
  }
};

extern "C" {

int fpx_serve_start(int device, const fpx_serve_config* cfg, fpx_server** out) {
  if (!out) return FPX_EINVAL;
  *out = nullptr;
  auto s = std::make_unique<fpx_server>();
  s->device = device;
  if (cfg) s->cfg = *cfg;
  if (s->cfg.hbm_budget_bytes == 0) {
    // a quarter of the device memory free at start, at most 32 GiB
    size_t free_b = 0, total_b = 0;
    if (cudaSetDevice(device) != cudaSuccess || cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      cudaGetLastError();
      free_b = size_t(32) << 30;
    }
    s->cfg.hbm_budget_bytes = std::min(free_b / 4, size_t(32) << 30);
  }
  if (s->cfg.max_batch_jobs == 0) s->cfg.max_batch_jobs = 4096;
  if (s->cfg.workers <= 0) s->cfg.workers = 6;
  if (s->cfg.workers < 2) s->cfg.workers = 2;
  // half the workers (at least one) for the large lane, the rest for the small lane
  s->small_workers = s->cfg.workers - std::max(1, s->cfg.workers / 2);
  if (s->cfg.repr != FPX_REPR_CANONICAL && s->cfg.repr != FPX_REPR_MONTGOMERY) return FPX_EINVAL;
  try {
    for (int w = 0; w < s->cfg.workers; ++w) s->engines.push_back(std::make_unique<fpx::Engine>(device, 0));
  } catch (const fpx::Error& e) {
    return e.code;
  } catch (...) {
    return FPX_ECUDA;
  }
  fpx_server* raw = s.get();
  for (int w = 0; w < s->cfg.workers; ++w) s->workers.emplace_back([raw, w] { raw->worker(w); });
  *out = s.release();
  return FPX_OK;
}

int fpx_serve_submit(fpx_server* srv, fpx_job* job, uint64_t* ticket) {
  if (!srv || !job || !ticket) return FPX_EINVAL;
  auto r = std::make_unique<Request>();
  r->job = job;
  r->bytes = fpx_serve_plan_bytes(job);
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> g(srv->mu);
    if (srv->stopping) return FPX_EINVAL;
    r->ticket = srv->next_ticket++;
    *ticket = r->ticket;
    srv->queue[lane_of(job)].push_back(r.get());
    srv->all.emplace(r->ticket, std::move(r));
    ++srv->stats.submitted;
  }
  srv->cv_work.notify_all();
  return FPX_OK;
}

int fpx_serve_poll(fpx_server* srv, uint64_t ticket, int wait, uint64_t* latency_ns) {
  if (!srv) return FPX_EINVAL;
  std::unique_lock<std::mutex> g(srv->mu);
  auto it = srv->all.find(ticket);
  if (it == srv->all.end()) return FPX_EINVAL;
  Request* r = it->second.get();
  if (!r->done) {
    if (!wait) return FPX_EPENDING;
    srv->cv_done.wait(g, [&] { return r->done; });
  }
  if (latency_ns)
    *latency_ns = (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(r->t_done - r->t_submit).count();
  const int st = r->job->status;
  srv->all.erase(it);
  return st;
}

int fpx_serve_stats_get(fpx_server* srv, fpx_serve_stats* out) {
  if (!srv || !out) return FPX_EINVAL;
  {
    std::lock_guard<std::mutex> g(srv->mu);
    *out = srv->stats;
  }
  out->device_pool_bytes = out->device_allocations = out->pool_flushes = 0;
  out->device_alloc_ns = out->device_alloc_ns_max = 0;
  out->host_allocs = out->host_alloc_ns = out->host_alloc_ns_max = 0;
  for (auto& e : srv->engines) {
    const fpx::Pool::Snapshot p = e->pool().snapshot();
    out->device_pool_bytes += p.cached_bytes + p.in_use_bytes;
    out->device_allocations += p.system_allocations;
    out->pool_flushes += p.flushes;
    out->device_alloc_ns += p.alloc_ns;
    out->device_alloc_ns_max = std::max<uint64_t>(out->device_alloc_ns_max, p.alloc_ns_max);
    out->host_allocs += e->host_allocs.load();
    out->host_alloc_ns += e->host_alloc_ns.load();
    out->host_alloc_ns_max = std::max<uint64_t>(out->host_alloc_ns_max, e->host_alloc_ns_max.load());
  }
  return FPX_OK;
}

int fpx_serve_stop(fpx_server* srv) {
  if (!srv) return FPX_EINVAL;
  {
    std::lock_guard<std::mutex> g(srv->mu);
    srv->stopping = true;
  }
  srv->cv_work.notify_all();
  for (auto& t : srv->workers) t.join();
  delete srv;
  return FPX_OK;
}

}  // extern "C"
