// server.cu -- served label propagation: a request loop that keeps graphs and
// label state in HBM, admits solves of mixed size and method against an HBM
// budget as they arrive, and batches the small classic ones into the
// persistent batched kernel.  The reference has no serving mode; this is
// built on the engine's own entry points (glp_graph_* / glp_run for one graph,
// glp_batch_* for many).
//
// Threads.  Callers submit from any thread.  Admission (FIFO, by an estimate
// of each request's device bytes against the budget) runs under one mutex on
// every submit and every completion.  Admitted requests go to one of two
// paths:
//   batched : classic, unweighted, every degree <= 4096, at most
//             batch_max_vertices vertices.  One batch thread runs rounds:
//             each round packs EVERY batched request admitted so far (up to
//             max_batch_graphs) into one glp_batch with per-request iteration
//             counts and runs them in one persistent launch; requests that
//             arrive meanwhile join the next round (continuous batching at
//             round granularity).
//   plain   : everything else (layered, SLPA, weighted, hubs, large graphs),
//             on plain_workers threads (default 1: one solve already fills
//             the GPU, and two contend), each with its own graph handles and
//             streams, so their work overlaps with the rounds on the device.
//             A worker takes the admitted request of the smallest expected
//             service time, aged by how long it has waited.
//   short   : one-graph requests expected below short_job_us have a worker
//             of their own, so that a small layered or SLPA solve does not
//             wait behind a long one; plain workers take them only when they
//             have nothing else.
// The batch thread and the short worker run on streams of the device's
// highest priority: the block scheduler dispatches their blocks ahead of the
// queued blocks of a long solve sharing the GPU.
// A request's host buffers (CSR in, labels out) must stay valid until it is
// done.  Results are exactly those of glp_run alone: the batched kernel
// reproduces glp_run(method 1) per graph, and the plain path is glp_run.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/glp.h"

namespace glp {
void set_error(const char* fmt, ...);
int graph_set_stream_priority(glp_graph* g, int priority);
int batch_set_stream_priority(glp_batch* b, int priority);
int ingest_edges(const int32_t* src, const int32_t* dst, int64_t count, int32_t n, int32_t on_device, uint32_t flags,
                 int32_t** d_off, int32_t** d_cols, int64_t* m, int32_t* d_old, cudaStream_t s);
}  // namespace glp

namespace {

constexpr int32_t kBatchMaxDegree = 4096;

// A graph uploaded once and kept in HBM for any number of requests.
struct Resident {
  int64_t id = 0;
  int32_t n = 0;
  int64_t m = 0;
  int32_t max_degree = 0;
  int32_t* d_off = nullptr;
  int32_t* d_cols = nullptr;
  int32_t* d_w = nullptr;
  int64_t bytes = 0;
  int refs = 0;          // requests admitted or waiting on it
  bool removed = false;  // freed once refs drops to 0
};

struct Request {
  int64_t id = 0;
  Resident* res = nullptr;  // the resident graph, or null for a host CSR
  const int32_t* offsets = nullptr;
  const int32_t* cols = nullptr;
  const int32_t* weights = nullptr;
  int32_t n = 0;
  int64_t m = 0;
  int32_t method = 1;
  glp_params params{};
  int32_t niter = 0;
  int32_t* labels = nullptr;
  int32_t max_degree = 0;
  bool batched = false;
  bool short_job = false;  // one-graph, expected below short_job_us
  int64_t bytes = 0;
  double cost_s = 0;  // expected service time, for shortest-job-first
  volatile int32_t cancel = 0;  // glp_server_cancel: stop (one-graph solve) or discard (batched round)
  // results
  int32_t status = GLP_EAGAIN;
  std::string error;
  glp_request_stats stats{};
};

using Clock = std::chrono::steady_clock;

}  // namespace

struct glp_server {
  glp_server_config cfg{};
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv_work;  // batch thread and plain workers wait here
  std::condition_variable cv_done;  // waiters on results
  std::deque<Request*> pending;     // submitted, not admitted (FIFO)
  std::deque<Request*> batch_q;     // admitted, batched path
  std::deque<Request*> plain_q;     // admitted, plain path
  std::deque<Request*> short_q;     // admitted, plain path, short jobs
  int high_priority = 0;            // the device's most urgent stream priority
  std::unordered_map<int64_t, std::unique_ptr<Request>> all;
  std::unordered_map<int64_t, std::unique_ptr<Resident>> graphs;
  std::unordered_set<int64_t> removed_graphs;  // ids whose cached handles must go
  int64_t next_id = 1;
  int64_t next_graph = 1;
  int64_t used_bytes = 0;
  int64_t in_flight = 0;            // admitted and not done
  bool stopping = false;
  std::vector<std::thread> threads;
  std::atomic<int64_t> rounds{0};
  // one-graph solves running on the worker threads: while one holds the
  // GPU, a batched round takes a grid sized to itself (it can start beside
  // the solve); otherwise every SM
  std::atomic<int> solves{0};

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

// Device bytes a request may hold while it runs (upper estimates); a
// request on a resident graph does not count the graph itself.
int64_t estimate_bytes(const Request& r) {
  const int64_t n = r.n, m = r.m;
  const int64_t csr = r.res ? 0 : 4 * (n + 1) + 4 * (m + 4) + (r.weights ? 4 * (m + 4) : 0);
  if (r.batched)  // (upload) + packed CSR (8 B offsets) + staging + labels x2 + order + slack
    return csr + 8 * (n + 1) + 4 * m + 4 * (n + 1) + 12 * n + (1 << 20);
  int64_t b = csr;
  b += 8 * n + 8 * n + 32 * n;                 // labels, volumes, plan and frontier lists
  b += 8 * m + (r.weights ? 8 * m : 0);        // hub gather/sort scratch (bounded by the edges)
  if (r.method == GLP_METHOD_SLPA) b += 4 * (int64_t)std::max(1, r.params.slpa_T) * n + 4 * n;
  return b + (64 << 20);
}

// Device bytes of a cached one-graph handle on a resident graph (its own CSR
// copy and plan; the per-request buffers are counted by the request).
int64_t handle_bytes(const Resident& g) {
  return 4 * (int64_t)(g.n + 1) + 4 * (g.m + 4) + (g.d_w ? 4 * (g.m + 4) : 0) + 40 * (int64_t)g.n + (16 << 20);
}

void free_resident(Resident* g) {
  cudaFree(g->d_off);
  cudaFree(g->d_cols);
  cudaFree(g->d_w);
  g->d_off = g->d_cols = g->d_w = nullptr;
}

// Caller holds s->mu.
void release_graph_locked(glp_server* s, Resident* g) {
  if (!g) return;
  if (--g->refs == 0 && g->removed) {
    s->used_bytes -= g->bytes;
    free_resident(g);
    s->graphs.erase(g->id);
  }
}

// Caller holds s->mu.
void finish_locked(glp_server* s, Request* r, int status, const char* err) {
  r->status = status;
  if (err) r->error = err;
  r->stats.done_s = s->now();
  r->stats.status = status;
  s->used_bytes -= r->bytes;
  s->in_flight--;
  release_graph_locked(s, r->res);
  r->res = nullptr;
}

void finish(glp_server* s, Request* r, int status, const char* err) {
  std::lock_guard<std::mutex> lk(s->mu);
  finish_locked(s, r, status, err);
}

// Moves pending requests that fit the budget to their path (FIFO: the head
// waits for room; nothing overtakes it).  Caller holds s->mu.
void admit_locked(glp_server* s) {
  bool any = false;
  while (!s->pending.empty()) {
    Request* r = s->pending.front();
    if (s->used_bytes + r->bytes > s->cfg.hbm_budget_bytes && s->in_flight > 0) break;
    s->pending.pop_front();
    s->used_bytes += r->bytes;
    s->in_flight++;
    r->stats.admit_s = s->now();
    (r->batched ? s->batch_q : r->short_job ? s->short_q : s->plain_q).push_back(r);
    any = true;
  }
  if (any) s->cv_work.notify_all();
}

bool idle_locked(const glp_server* s) { return s->stopping && s->pending.empty() && s->in_flight == 0; }

// One-graph solves with a handle per resident graph: plans and buffers are
// built once and reused by later requests on that graph.  Each worker thread
// owns one.
struct OneGraphRunner {
  struct Cached {
    glp_graph* g;
    int64_t bytes;
  };
  glp_server* s;
  std::unordered_map<int64_t, Cached> cache;
  bool urgent = false;  // handles on the device's highest stream priority
  bool counted = false;  // a worker's runner: its solves show in glp_server::solves

  void drop(int64_t id) {
    auto it = cache.find(id);
    if (it == cache.end()) return;
    glp_graph_destroy(it->second.g);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->used_bytes -= it->second.bytes;
    }
    cache.erase(it);
  }
  // Caller holds s->mu: handles of removed graphs to drop outside the lock.
  std::vector<int64_t> stale_locked() const {
    std::vector<int64_t> out;
    for (auto& kv : cache)
      if (s->removed_graphs.count(kv.first)) out.push_back(kv.first);
    return out;
  }
  void clear() {
    for (auto& kv : cache) {
      glp_graph_destroy(kv.second.g);
      std::lock_guard<std::mutex> lk(s->mu);
      s->used_bytes -= kv.second.bytes;
    }
    cache.clear();
  }
  // Solves r with glp_run and finishes it.
  void run(Request* r) {
    glp_graph* g = nullptr;
    bool transient = true;
    int rc = GLP_OK;
    if (r->res) {
      auto it = cache.find(r->res->id);
      if (it != cache.end()) {
        g = it->second.g;
      } else {
        rc = glp_graph_create(r->res->d_off, r->res->d_cols, r->res->d_w, r->res->n, r->res->m, 1, &g);
        if (rc == GLP_OK && urgent && (rc = glp::graph_set_stream_priority(g, s->high_priority)) != GLP_OK) {
          glp_graph_destroy(g);
          g = nullptr;
        }
        if (rc == GLP_OK) {
          const int64_t hb = handle_bytes(*r->res);
          cache.emplace(r->res->id, Cached{g, hb});
          std::lock_guard<std::mutex> lk(s->mu);
          s->used_bytes += hb;
        }
      }
      transient = false;
    } else {
      rc = glp_graph_create(r->offsets, r->cols, r->weights, r->n, r->m, 0, &g);
      if (rc == GLP_OK && urgent) rc = glp::graph_set_stream_priority(g, s->high_priority);
    }
    if (rc == GLP_OK && r->cancel) {
      glp::set_error("cancelled before it started");
      rc = GLP_ECANCELED;
    }
    if (rc == GLP_OK) {
      glp_outputs out{};
      out.labels = r->labels;
      glp_graph_set_cancel_flag(g, &r->cancel);
      if (counted) s->solves.fetch_add(1);
      rc = glp_run(g, r->method, &r->params, r->niter, &out, nullptr, nullptr, nullptr);
      if (counted) s->solves.fetch_sub(1);
      glp_graph_set_cancel_flag(g, nullptr);
    }
    const std::string err = rc ? glp_last_error() : std::string();
    if (transient) glp_graph_destroy(g);
    finish(s, r, rc, rc ? err.c_str() : nullptr);
  }
};

// A plain worker serves plain_q, and short_q when plain_q is empty; the
// short worker (short_lane) serves short_q only, on urgent streams.
void plain_worker(glp_server* s, bool short_lane) {
  cudaSetDevice(s->cfg.device);
  OneGraphRunner one{s, {}, short_lane, true};
  for (;;) {
    Request* r = nullptr;
    std::vector<int64_t> stale;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      auto has_work = [&] { return !s->short_q.empty() || (!short_lane && !s->plain_q.empty()); };
      s->cv_work.wait(lk, [&] { return has_work() || idle_locked(s); });
      stale = one.stale_locked();
      if (!has_work()) {
        lk.unlock();
        one.clear();
        return;
      }
      // shortest expected job first, aged by its wait so none starves
      std::deque<Request*>& q = (short_lane || s->plain_q.empty()) ? s->short_q : s->plain_q;
      const double now = s->now();
      auto best = q.begin();
      for (auto it = q.begin(); it != q.end(); ++it)
        if ((*it)->cost_s - (now - (*it)->stats.admit_s) < (*best)->cost_s - (now - (*best)->stats.admit_s)) best = it;
      r = *best;
      q.erase(best);
      r->stats.start_s = now;
      r->stats.path = 0;
    }
    for (int64_t id : stale) one.drop(id);
    one.run(r);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      admit_locked(s);
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
}

void batch_worker(glp_server* s) {
  cudaSetDevice(s->cfg.device);
  std::vector<int32_t> packed;
  cudaStream_t up = nullptr;  // uploads of host CSRs, finished before packing
  cudaStreamCreateWithFlags(&up, cudaStreamNonBlocking);
  glp_batch* b = nullptr;     // kept across rounds: repacking reuses its buffers
  // host CSRs of a round are uploaded into one grow-only staging buffer: no
  // allocation or free per round (a free waits for every stream of the
  // device, the one-graph solves of the plain workers included)
  int32_t* stage = nullptr;
  size_t stage_cap = 0;  // int32 elements
  // With lone_one_graph set, a round of one request runs as a one-graph
  // solve instead.  By default it rides the batched kernel like any round:
  // one launch on a grid sized to the round (measured on the served
  // workload at 50 req/s: p50 3.0 ms batched, 6.5 ms as one-graph solves,
  // whose ~100 launches a request each queue behind a long solve's blocks).
  OneGraphRunner one{s, {}, true};
  for (;;) {
    std::vector<Request*> round;
    std::vector<int64_t> stale;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] { return !s->batch_q.empty() || idle_locked(s); });
      stale = one.stale_locked();
      if (s->batch_q.empty()) {
        lk.unlock();
        if (up) cudaStreamDestroy(up);
        cudaFree(stage);
        glp_batch_destroy(b);
        one.clear();
        return;
      }
      while (!s->batch_q.empty() && (int32_t)round.size() < s->cfg.max_batch_graphs) {
        round.push_back(s->batch_q.front());
        s->batch_q.pop_front();
      }
      const double t = s->now();
      for (Request* r : round) {
        r->stats.start_s = t;
        r->stats.path = (round.size() > 1 || s->cfg.lone_one_graph <= 0) ? 1 : 0;
        r->stats.batch_graphs = (int32_t)round.size();
      }
    }
    for (int64_t id : stale) one.drop(id);
    if (round.size() == 1 && s->cfg.lone_one_graph > 0) {
      one.run(round[0]);
      {
        std::lock_guard<std::mutex> lk(s->mu);
        admit_locked(s);
      }
      s->cv_done.notify_all();
      s->cv_work.notify_all();
      continue;
    }
    // pack in order of iteration count (the batch wants them non-decreasing);
    // host CSRs are uploaded first so the whole round packs device to device
    std::stable_sort(round.begin(), round.end(), [](const Request* a, const Request* b) { return a->niter < b->niter; });
    const size_t G = round.size();
    std::vector<const int32_t*> offs(G), cols(G);
    std::vector<int32_t> ns(G), its(G);
    std::vector<int64_t> ms(G);
    int64_t total = 0;
    int rc = GLP_OK;
    // staging layout: per host request, offsets then columns, each segment
    // starting on a 64-element (256-byte) boundary
    auto seg = [](size_t e) { return (e + 63) & ~(size_t)63; };
    size_t need = 0;
    for (Request* r : round)
      if (!r->res) need += seg((size_t)r->n + 1) + seg((size_t)std::max<int64_t>(r->m, 1));
    if (need > stage_cap) {
      cudaFree(stage);
      stage = nullptr;
      stage_cap = 0;
      const size_t want = need + need / 4;
      if (cudaMalloc(&stage, sizeof(int32_t) * want) == cudaSuccess) {
        stage_cap = want;
      } else {
        glp::set_error("staging a round's host CSRs: out of device memory");
        rc = GLP_ENOMEM;
      }
    }
    size_t at = 0;
    bool uploaded = false;
    for (size_t i = 0; i < G; ++i) {
      Request* r = round[i];
      ns[i] = r->n;
      ms[i] = r->m;
      its[i] = r->niter;
      total += r->n;
      if (r->res) {
        offs[i] = r->res->d_off;
        cols[i] = r->res->d_cols;
        continue;
      }
      if (rc != GLP_OK) continue;
      int32_t* d_o = stage + at;
      at += seg((size_t)r->n + 1);
      int32_t* d_c = stage + at;
      at += seg((size_t)std::max<int64_t>(r->m, 1));
      if (cudaMemcpyAsync(d_o, r->offsets, sizeof(int32_t) * ((size_t)r->n + 1), cudaMemcpyHostToDevice, up) !=
              cudaSuccess ||
          (r->m &&
           cudaMemcpyAsync(d_c, r->cols, sizeof(int32_t) * (size_t)r->m, cudaMemcpyHostToDevice, up) != cudaSuccess)) {
        glp::set_error("uploading a request's CSR failed");
        rc = GLP_ECUDA;
      }
      uploaded = true;
      offs[i] = d_o;
      cols[i] = d_c;
    }
    if (rc == GLP_OK && uploaded && cudaStreamSynchronize(up) != cudaSuccess) {
      glp::set_error("uploading a request's CSR failed");
      rc = GLP_ECUDA;
    }
    if (rc == GLP_OK && b) {
      rc = glp_batch_repack(b, (int32_t)G, offs.data(), cols.data(), ns.data(), ms.data(), 1, its.data());
    } else if (rc == GLP_OK) {
      rc = glp_batch_create_ex((int32_t)G, offs.data(), cols.data(), ns.data(), ms.data(), 1, its.data(), &b);
      if (rc == GLP_OK) rc = glp::batch_set_stream_priority(b, s->high_priority);
    }
    if (rc == GLP_OK) {
      packed.resize((size_t)std::max<int64_t>(total, 1));
      // while a one-graph solve of a worker thread holds the GPU, a grid
      // sized to the round (one CTA per 8192 vertices, at least 8), whose
      // CTAs can all become resident beside the solve's blocks; on an
      // otherwise idle GPU one CTA per 1024 vertices (a lone graph of 10k-100k
      // vertices on eight CTAs would use a twentieth of the GPU; on every SM
      // it would hold the whole GPU, and a short solve arriving meanwhile
      // would wait for the round)
      glp_params bp;
      glp_params_default(&bp);
      bp.batch_blocks = (int32_t)std::min<int64_t>(
          INT32_MAX, std::max<int64_t>(8, s->solves.load() > 0 ? (total + 8191) / 8192 : (total + 1023) / 1024));
      rc = glp_batch_run(b, &bp, GLP_BATCH_OWN_ITERATIONS, packed.data(), 0, nullptr, nullptr);
    }
    const std::string err = rc ? glp_last_error() : std::string();
    s->rounds++;
    int64_t base = 0;
    for (Request* r : round) {
      if (r->cancel) {  // cancelled while its round ran: the result is discarded
        base += r->n;
        finish(s, r, GLP_ECANCELED, "cancelled during its batched round");
        continue;
      }
      if (rc == GLP_OK && r->n) std::memcpy(r->labels, packed.data() + base, sizeof(int32_t) * (size_t)r->n);
      base += r->n;
      finish(s, r, rc, rc ? err.c_str() : nullptr);
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);
      admit_locked(s);
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
}

int32_t host_max_degree(const int32_t* off, int32_t n) {
  int32_t d = 0;
  for (int32_t v = 0; v < n; ++v) d = std::max(d, off[v + 1] - off[v]);
  return d;
}

// Builds and enqueues a request.  Caller holds nothing.
int submit_request(glp_server* s, std::unique_ptr<Request> r, int64_t* id) {
  r->batched = r->method == GLP_METHOD_CLASSIC && !(r->res ? r->res->d_w : r->weights) &&
               r->max_degree <= kBatchMaxDegree && r->n <= s->cfg.batch_max_vertices && !r->params.async;
  r->bytes = estimate_bytes(*r);
  // about 1e10 edge visits per second for a one-graph solve, plus a fixed part
  const int64_t iters = (int64_t)r->niter * (r->method == GLP_METHOD_LAYERED ? std::max(1, r->params.nlayers) : 1);
  r->cost_s = 1e-3 + (double)(r->m + r->n) * (double)iters * 1e-10;
  r->short_job = !r->batched && s->cfg.short_job_us > 0 && r->cost_s * 1e6 < (double)s->cfg.short_job_us;
  if (r->bytes > s->cfg.hbm_budget_bytes) {
    glp::set_error("request needs about %lld bytes, above the server's HBM budget", (long long)r->bytes);
    return GLP_ENOMEM;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stopping) {
    glp::set_error("server is stopping");
    return GLP_ECANCELED;
  }
  if (r->res) {
    if (r->res->removed) {
      glp::set_error("graph %lld was removed", (long long)r->res->id);
      return GLP_EINVAL;
    }
    r->res->refs++;
  }
  r->id = s->next_id++;
  r->stats.submit_s = s->now();
  *id = r->id;
  s->pending.push_back(r.get());
  s->all.emplace(r->id, std::move(r));
  admit_locked(s);
  return GLP_OK;
}

int copy_params(Request* r, const glp_params* p) {
  if (p) {
    if (p->struct_size != (int32_t)sizeof(glp_params)) {
      glp::set_error("glp_params.struct_size mismatch");
      return GLP_EINVAL;
    }
    r->params = *p;
  } else {
    glp_params_default(&r->params);
  }
  return GLP_OK;
}

}  // namespace

using glp::set_error;

extern "C" {

int glp_server_config_default(glp_server_config* c) {
  if (!c) {
    set_error("config is NULL");
    return GLP_EINVAL;
  }
  std::memset(c, 0, sizeof *c);
  c->struct_size = (int32_t)sizeof(glp_server_config);
  c->device = -1;
  c->hbm_budget_bytes = 150ll * 1000 * 1000 * 1000;
  c->max_batch_graphs = 4096;
  c->plain_workers = 1;
  c->batch_max_vertices = 1 << 22;
  c->short_job_us = 20000;
  return GLP_OK;
}

int glp_server_start(const glp_server_config* cfg, glp_server** out) {
  if (!out) {
    set_error("out is NULL");
    return GLP_EINVAL;
  }
  *out = nullptr;
  glp_server_config c;
  glp_server_config_default(&c);
  if (cfg) {
    if (cfg->struct_size != (int32_t)sizeof(glp_server_config)) {
      set_error("glp_server_config.struct_size mismatch");
      return GLP_EINVAL;
    }
    c = *cfg;
  }
  if (c.hbm_budget_bytes <= 0 || c.max_batch_graphs <= 0 || c.plain_workers <= 0 || c.plain_workers > 64) {
    set_error("bad server configuration");
    return GLP_EINVAL;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    set_error("no usable CUDA device");
    return GLP_ENODEV;
  }
  if (c.device < 0) cudaGetDevice(&c.device);
  if (c.device >= count) {
    set_error("device %d does not exist", c.device);
    return GLP_EINVAL;
  }
  if (c.short_job_us == 0) c.short_job_us = 20000;
  std::unique_ptr<glp_server> s(new glp_server());
  s->cfg = c;
  s->t0 = Clock::now();
  int least = 0, greatest = 0;
  if (cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess) s->high_priority = greatest;
  s->threads.emplace_back(batch_worker, s.get());
  for (int i = 0; i < c.plain_workers; ++i) s->threads.emplace_back(plain_worker, s.get(), false);
  if (c.short_job_us > 0) s->threads.emplace_back(plain_worker, s.get(), true);
  *out = s.release();
  return GLP_OK;
}

int glp_server_submit(glp_server* s, const int32_t* offsets, const int32_t* cols, const int32_t* weights, int32_t n,
                      int64_t m, int32_t method, const glp_params* p, int32_t niter, int32_t* labels_out,
                      int64_t* id) {
  if (!s || !offsets || (m > 0 && !cols) || n < 0 || m < 0 || niter < 0 || (n > 0 && !labels_out) || !id) {
    set_error("bad request arguments");
    return GLP_EINVAL;
  }
  if (method < GLP_METHOD_CLASSIC || method > GLP_METHOD_USER) {
    set_error("method %d not in 1..4", method);
    return GLP_ENOTSUP;
  }
  std::unique_ptr<Request> r(new Request());
  r->offsets = offsets;
  r->cols = cols;
  r->weights = weights;
  r->n = n;
  r->m = m;
  r->method = method;
  r->niter = niter;
  r->labels = labels_out;
  int rc = copy_params(r.get(), p);
  if (rc) return rc;
  r->max_degree = host_max_degree(offsets, n);
  return submit_request(s, std::move(r), id);
}

int glp_server_add_graph(glp_server* s, const int32_t* offsets, const int32_t* cols, const int32_t* weights, int32_t n,
                         int64_t m, int32_t on_device, int64_t* graph_id) {
  if (!s || !offsets || (m > 0 && !cols) || n < 0 || m < 0 || m > INT32_MAX || !graph_id) {
    set_error("bad graph arguments");
    return GLP_EINVAL;
  }
  std::unique_ptr<Resident> g(new Resident());
  g->n = n;
  g->m = m;
  g->bytes = 4 * (int64_t)(n + 1) + 4 * std::max<int64_t>(m, 1) + (weights ? 4 * std::max<int64_t>(m, 1) : 0);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->used_bytes + g->bytes > s->cfg.hbm_budget_bytes) {
      set_error("adding the graph would exceed the server's HBM budget");
      return GLP_ENOMEM;
    }
    s->used_bytes += g->bytes;  // reserved while uploading
  }
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  cudaError_t e = cudaSetDevice(s->cfg.device);
  std::vector<int32_t> hoff;
  if (e == cudaSuccess) e = cudaMalloc(&g->d_off, sizeof(int32_t) * ((size_t)n + 1));
  if (e == cudaSuccess) e = cudaMalloc(&g->d_cols, sizeof(int32_t) * (size_t)std::max<int64_t>(m, 1));
  if (e == cudaSuccess && weights) e = cudaMalloc(&g->d_w, sizeof(int32_t) * (size_t)std::max<int64_t>(m, 1));
  if (e == cudaSuccess) e = cudaMemcpy(g->d_off, offsets, sizeof(int32_t) * ((size_t)n + 1), kind);
  if (e == cudaSuccess && m) e = cudaMemcpy(g->d_cols, cols, sizeof(int32_t) * (size_t)m, kind);
  if (e == cudaSuccess && m && weights) e = cudaMemcpy(g->d_w, weights, sizeof(int32_t) * (size_t)m, kind);
  if (e == cudaSuccess) {  // after the copies above on the same stream: they are done on return
    hoff.resize((size_t)n + 1);
    e = cudaMemcpy(hoff.data(), g->d_off, sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyDeviceToHost);
  }
  if (e != cudaSuccess) {
    free_resident(g.get());
    std::lock_guard<std::mutex> lk(s->mu);
    s->used_bytes -= g->bytes;
    set_error("uploading the graph failed: %s", cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? GLP_ENOMEM : GLP_ECUDA;
  }
  for (int32_t v = 0; v < n; ++v)
    if (hoff[v + 1] < hoff[v]) {
      free_resident(g.get());
      std::lock_guard<std::mutex> lk(s->mu);
      s->used_bytes -= g->bytes;
      set_error("offsets not monotone");
      return GLP_EINVAL;
    }
  g->max_degree = host_max_degree(hoff.data(), n);
  std::lock_guard<std::mutex> lk(s->mu);
  g->id = s->next_graph++;
  *graph_id = g->id;
  s->graphs.emplace(g->id, std::move(g));
  return GLP_OK;
}

int glp_server_add_edges(glp_server* s, const int32_t* src, const int32_t* dst, int64_t count, int32_t n,
                         int32_t on_device, uint32_t flags, int32_t* old_id, int64_t* graph_id) {
  if (!s || !graph_id) {
    set_error("bad graph arguments");
    return GLP_EINVAL;
  }
  // the CSR is built on the device; its size is known only afterwards, so the
  // budget is checked against the edge count's bound first
  const int64_t bound = 4 * ((int64_t)n + 1) + 4 * std::max<int64_t>(((flags & GLP_EDGES_DIRECTED) ? 1 : 2) * count, 1);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->used_bytes + bound > s->cfg.hbm_budget_bytes) {
      set_error("adding the graph would exceed the server's HBM budget");
      return GLP_ENOMEM;
    }
    s->used_bytes += bound;  // reserved while building
  }
  std::unique_ptr<Resident> g(new Resident());
  cudaStream_t st = nullptr;
  int rc = cudaSetDevice(s->cfg.device) == cudaSuccess && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) ==
                                                                cudaSuccess
               ? GLP_OK
               : GLP_ECUDA;
  int32_t* d_old = nullptr;
  if (!rc && old_id) {
    if (on_device) d_old = old_id;
    else if (cudaMalloc(&d_old, sizeof(int32_t) * (size_t)std::max(n, 1)) != cudaSuccess) rc = GLP_ENOMEM;
  }
  if (!rc) rc = glp::ingest_edges(src, dst, count, n, on_device, flags, &g->d_off, &g->d_cols, &g->m, d_old, st);
  if (!rc && old_id && !on_device &&
      (cudaMemcpy(old_id, d_old, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess))
    rc = GLP_ECUDA;
  std::vector<int32_t> hoff;
  if (!rc) {
    hoff.resize((size_t)n + 1);
    if (cudaMemcpy(hoff.data(), g->d_off, sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = GLP_ECUDA;
  }
  if (old_id && !on_device && d_old) cudaFree(d_old);
  if (st) cudaStreamDestroy(st);
  std::lock_guard<std::mutex> lk(s->mu);
  s->used_bytes -= bound;
  if (rc) {
    free_resident(g.get());
    if (rc == GLP_ECUDA) set_error("building the graph on the device failed");
    return rc;
  }
  g->n = n;
  g->bytes = 4 * (int64_t)(n + 1) + 4 * std::max<int64_t>(g->m, 1);
  g->max_degree = host_max_degree(hoff.data(), n);
  s->used_bytes += g->bytes;
  g->id = s->next_graph++;
  *graph_id = g->id;
  s->graphs.emplace(g->id, std::move(g));
  return GLP_OK;
}

int glp_server_submit_graph(glp_server* s, int64_t graph_id, int32_t method, const glp_params* p, int32_t niter,
                            int32_t* labels_out, int64_t* id) {
  if (!s || niter < 0 || !id) {
    set_error("bad request arguments");
    return GLP_EINVAL;
  }
  if (method < GLP_METHOD_CLASSIC || method > GLP_METHOD_USER) {
    set_error("method %d not in 1..4", method);
    return GLP_ENOTSUP;
  }
  std::unique_ptr<Request> r(new Request());
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->graphs.find(graph_id);
    if (it == s->graphs.end() || it->second->removed) {
      set_error("unknown graph %lld", (long long)graph_id);
      return GLP_EINVAL;
    }
    r->res = it->second.get();
  }
  if (r->res->n > 0 && !labels_out) {
    set_error("labels_out is NULL");
    return GLP_EINVAL;
  }
  r->n = r->res->n;
  r->m = r->res->m;
  r->method = method;
  r->niter = niter;
  r->labels = labels_out;
  r->max_degree = r->res->max_degree;
  int rc = copy_params(r.get(), p);
  if (rc) return rc;
  return submit_request(s, std::move(r), id);
}

int glp_server_remove_graph(glp_server* s, int64_t graph_id) {
  if (!s) {
    set_error("server is NULL");
    return GLP_EINVAL;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->graphs.find(graph_id);
  if (it == s->graphs.end() || it->second->removed) {
    set_error("unknown graph %lld", (long long)graph_id);
    return GLP_EINVAL;
  }
  Resident* g = it->second.get();
  g->removed = true;
  s->removed_graphs.insert(graph_id);
  if (g->refs == 0) {
    g->refs = 1;
    release_graph_locked(s, g);
  }
  s->cv_work.notify_all();
  return GLP_OK;
}

static int report(glp_server* s, Request* r, glp_request_stats* st) {
  if (st) *st = r->stats;
  if (r->status != GLP_OK && r->status != GLP_EAGAIN) set_error("request %lld: %s", (long long)r->id, r->error.c_str());
  (void)s;
  return r->status;
}

int glp_server_poll(glp_server* s, int64_t id, glp_request_stats* st) {
  if (!s) {
    set_error("server is NULL");
    return GLP_EINVAL;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) {
    set_error("unknown request %lld", (long long)id);
    return GLP_EINVAL;
  }
  return report(s, it->second.get(), st);
}

int glp_server_wait(glp_server* s, int64_t id, int32_t timeout_ms, glp_request_stats* st) {
  if (!s) {
    set_error("server is NULL");
    return GLP_EINVAL;
  }
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) {
    set_error("unknown request %lld", (long long)id);
    return GLP_EINVAL;
  }
  Request* r = it->second.get();
  auto done = [&] { return r->status != GLP_EAGAIN; };
  if (timeout_ms < 0) {
    s->cv_done.wait(lk, done);
  } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) {
    set_error("request %lld not done within %d ms", (long long)id, timeout_ms);
    return GLP_ETIMEOUT;
  }
  return report(s, r, st);
}

int glp_server_release(glp_server* s, int64_t id) {
  if (!s) {
    set_error("server is NULL");
    return GLP_EINVAL;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end() || it->second->status == GLP_EAGAIN) {
    set_error("request %lld is unknown or not done", (long long)id);
    return GLP_EINVAL;
  }
  s->all.erase(it);
  return GLP_OK;
}

int glp_server_cancel(glp_server* s, int64_t id) {
  if (!s) {
    set_error("server is NULL");
    return GLP_EINVAL;
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) {
      set_error("unknown request %lld", (long long)id);
      return GLP_EINVAL;
    }
    Request* r = it->second.get();
    if (r->status != GLP_EAGAIN) return GLP_OK;  // already finished: its result stands
    r->cancel = 1;
    auto take = [&](std::deque<Request*>& q) {
      auto f = std::find(q.begin(), q.end(), r);
      if (f == q.end()) return false;
      q.erase(f);
      return true;
    };
    if (take(s->pending)) {  // never admitted: it holds no budget
      r->status = GLP_ECANCELED;
      r->error = "cancelled before admission";
      r->stats.done_s = s->now();
      r->stats.status = GLP_ECANCELED;
      release_graph_locked(s, r->res);
      r->res = nullptr;
    } else if (take(s->batch_q) || take(s->plain_q) || take(s->short_q)) {
      finish_locked(s, r, GLP_ECANCELED, "cancelled before it started");
    }
    // otherwise it is running: its worker sees r->cancel
    admit_locked(s);
  }
  s->cv_done.notify_all();
  s->cv_work.notify_all();
  return GLP_OK;
}

int glp_server_info(glp_server* s, int64_t* pending, int64_t* in_flight, int64_t* used_bytes, int64_t* rounds) {
  if (!s) {
    set_error("server is NULL");
    return GLP_EINVAL;
  }
  std::lock_guard<std::mutex> lk(s->mu);
  if (pending) *pending = (int64_t)s->pending.size();
  if (in_flight) *in_flight = s->in_flight;
  if (used_bytes) *used_bytes = s->used_bytes;
  if (rounds) *rounds = s->rounds.load();
  return GLP_OK;
}

int glp_server_stop(glp_server* s) {
  if (!s) return GLP_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->threads) t.join();
  for (auto& kv : s->graphs) free_resident(kv.second.get());
  delete s;
  return GLP_OK;
}

}  // extern "C"
