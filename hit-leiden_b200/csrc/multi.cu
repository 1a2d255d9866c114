// multi.cu — many graphs on one GPU: the batching and serving forms of the
// update path (host-side executors over the per-graph C ABI).
//
// Every graph handle owns its CUDA stream, its engine state and its device
// memory, so updates of different graphs are independent: run from different
// host threads, their kernels and their host round trips (the few scalar
// read-backs each stage needs) overlap on the GPU.  A small graph's batch is
// bound by launch and round-trip latency, not by the GPU; running many of
// them at once fills the device.  Results are those of each graph's batch run
// alone: graphs share nothing but the device.
//
//   hl_apply_batches  one batch per graph, all graphs at once (batching form);
//   hl_server_*       a request loop (serving form): requests for resident
//                     graphs are admitted against an HBM budget, requests
//                     for a graph that arrive while it is busy are coalesced
//                     into its next batch (in arrival order), and different
//                     graphs are updated concurrently by a pool of workers.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <limits>
#include <memory>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/hl.h"

namespace hl {
hl_status apply_on_handle(hl_graph* g, const uint32_t* src, const uint32_t* dst, const double* w,
                          uint64_t k, hl_batch_stats* stats, std::string* err);
uint64_t handle_device_bytes(const hl_graph* g);
}  // namespace hl

void hl_set_error_message(const std::string& m);

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// ---------------------------------------------------------------------------
// Serving
// ---------------------------------------------------------------------------
struct Request {
  uint64_t id;
  uint32_t graph;
  std::vector<uint32_t> src, dst;
  std::vector<double> w;  // empty = all +1.0
  uint64_t estimate;      // bytes reserved against the budget while in flight
  Clock::time_point t_submit, t_admit;
};

struct LevelCtx;  // per-graph context of the per-level output trampoline

struct GraphSlot {
  hl_graph* g = nullptr;
  std::unique_ptr<LevelCtx> lvl;  // stable address handed to the handle's callback
  std::deque<Request> pending;  // admitted, waiting for the graph
  bool busy = false;
  bool queued = false;          // in the ready list
  uint64_t batches = 0;         // batches applied (per-graph sequence number)
  uint64_t bytes = 0;           // device bytes the handle holds (refreshed by
                                // the worker that last updated it)
};

// The graph and batch a handle's level callback belongs to, and when its
// level 0 was ready.
struct LevelCtx {
  hl_server* server = nullptr;
  uint32_t graph = 0;
  uint64_t batch_id = 0;
  bool have_l0 = false;
  Clock::time_point t_l0;
};

void level_trampoline(void* user, uint32_t level, uint64_t count, const uint32_t* nodes,
                      const uint32_t* ids);

}  // namespace

struct hl_server {
  std::mutex mu;
  std::condition_variable cv_work;  // workers: a graph became ready / shutdown
  std::condition_variable cv_done;  // pollers / drain: something completed
  std::vector<GraphSlot> graphs;
  std::deque<uint32_t> ready;       // graphs with admitted work, not busy
  std::deque<Request> backlog;      // submitted, not yet admitted (FIFO)
  std::vector<hl_request_done> done;
  std::vector<std::thread> workers;
  uint64_t budget = 0;              // 0 = no admission control
  uint64_t reserved = 0;            // estimates of admitted, unfinished requests
  uint64_t next_id = 1;
  uint64_t next_batch = 1;
  uint64_t outstanding = 0;         // submitted, not completed
  uint64_t bytes_per_edge = 512;
  uint32_t max_coalesce = 0;        // requests per batch at most (0 = all pending)
  bool stop = false;
  std::atomic<hl_server_level_fn> level_fn{nullptr};  // per-level output, if set
  std::atomic<void*> level_user{nullptr};

  uint64_t resident_bytes() const {
    uint64_t s = 0;
    for (const GraphSlot& x : graphs) s += x.bytes;
    return s;
  }

  // Move backlog requests into their graphs' queues while the budget allows
  // (caller holds mu).  A request that cannot fit even with nothing else in
  // flight is completed with HL_ERR_OUT_OF_MEMORY.
  void admit_locked() {
    while (!backlog.empty()) {
      Request& r = backlog.front();
      if (budget) {
        const uint64_t used = resident_bytes() + reserved;
        if (used + r.estimate > budget) {
          if (reserved == 0) {
            hl_request_done d{};
            d.request_id = r.id;
            d.graph = r.graph;
            d.status = (int32_t)HL_ERR_OUT_OF_MEMORY;
            d.edges = r.src.size();
            d.latency_ms = ms_between(r.t_submit, Clock::now());
            done.push_back(d);
            --outstanding;
            backlog.pop_front();
            cv_done.notify_all();
            continue;
          }
          return;  // wait for in-flight work to finish
        }
      }
      reserved += r.estimate;
      r.t_admit = Clock::now();
      GraphSlot& gs = graphs[r.graph];
      const uint32_t gid = r.graph;
      gs.pending.push_back(std::move(r));
      backlog.pop_front();
      if (!gs.busy && !gs.queued) {
        gs.queued = true;
        ready.push_back(gid);
        cv_work.notify_one();
      }
    }
  }

  void worker_loop() {
    std::vector<uint32_t> src, dst;
    std::vector<double> w;
    for (;;) {
      std::vector<Request> batch;
      uint32_t gid = 0;
      uint64_t batch_id = 0, seq = 0;
      hl_graph* g = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_work.wait(lk, [&] { return stop || !ready.empty(); });
        if (ready.empty()) return;  // stop requested and nothing left
        gid = ready.front();
        ready.pop_front();
        GraphSlot& gs = graphs[gid];
        gs.queued = false;
        gs.busy = true;
        while (!gs.pending.empty() &&  // coalesce what was admitted so far
               (max_coalesce == 0 || batch.size() < max_coalesce)) {
          batch.push_back(std::move(gs.pending.front()));
          gs.pending.pop_front();
        }
        batch_id = next_batch++;
        seq = ++gs.batches;
        g = gs.g;
      }
      // one batch: the requests' edges in arrival order
      src.clear();
      dst.clear();
      w.clear();
      bool any_w = false;
      for (const Request& r : batch) any_w |= !r.w.empty();
      for (const Request& r : batch) {
        src.insert(src.end(), r.src.begin(), r.src.end());
        dst.insert(dst.end(), r.dst.begin(), r.dst.end());
        if (any_w) {
          if (r.w.empty()) w.insert(w.end(), r.src.size(), 1.0);
          else w.insert(w.end(), r.w.begin(), r.w.end());
        }
      }
      LevelCtx* lc = nullptr;
      {
        std::lock_guard<std::mutex> lk(mu);
        lc = graphs[gid].lvl.get();
      }
      lc->batch_id = batch_id;
      lc->have_l0 = false;
      if (level_fn.load()) hl_set_level_callback(g, level_trampoline, lc);
      else hl_set_level_callback(g, nullptr, nullptr);
      const Clock::time_point t0 = Clock::now();
      hl_batch_stats st{};
      std::string err;
      const hl_status rc = hl::apply_on_handle(g, src.data(), dst.data(),
                                               any_w ? w.data() : nullptr, src.size(), &st, &err);
      const Clock::time_point t1 = Clock::now();
      const uint64_t held = hl::handle_device_bytes(g);  // this worker owns g here
      {
        std::lock_guard<std::mutex> lk(mu);
        graphs[gid].bytes = held;
        for (const Request& r : batch) {
          hl_request_done d{};
          d.request_id = r.id;
          d.graph = gid;
          d.status = (int32_t)rc;
          d.edges = r.src.size();
          d.batch_id = batch_id;
          d.batch_seq = seq;
          d.batch_requests = (uint32_t)batch.size();
          d.batch_edges = src.size();
          d.changed = st.changed;
          d.modularity = st.modularity;
          d.queue_ms = ms_between(r.t_submit, t0);
          d.service_ms = ms_between(t0, t1);
          d.latency_ms = ms_between(r.t_submit, t1);
          d.level0_ms = lc->have_l0 ? ms_between(r.t_submit, lc->t_l0)
                                    : std::numeric_limits<double>::quiet_NaN();
          done.push_back(d);
          reserved -= r.estimate;
          --outstanding;
        }
        GraphSlot& gs = graphs[gid];
        gs.busy = false;
        if (!gs.pending.empty() && !gs.queued) {
          gs.queued = true;
          ready.push_back(gid);
          cv_work.notify_one();
        }
        admit_locked();
      }
      cv_done.notify_all();
      (void)err;
    }
  }
};

namespace {

void level_trampoline(void* user, uint32_t level, uint64_t count, const uint32_t* nodes,
                      const uint32_t* ids) {
  LevelCtx* c = static_cast<LevelCtx*>(user);
  if (level == 0) {
    c->t_l0 = Clock::now();
    c->have_l0 = true;
  }
  hl_server_level_fn fn = c->server->level_fn.load();
  if (fn) fn(c->server->level_user.load(), c->graph, c->batch_id, level, count, nodes, ids);
}

#define HLM_TRY(...)                   \
  try {                                \
    __VA_ARGS__;                       \
    hl_set_error_message("");          \
    return HL_OK;                      \
  } catch (const std::exception& e) {  \
    hl_set_error_message(e.what());    \
    return HL_ERR_INVALID_INPUT;       \
  }

struct Bad : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void need(bool ok, const char* msg) {
  if (!ok) throw Bad(msg);
}

}  // namespace

extern "C" {

HL_API hl_status hl_apply_batches(hl_graph* const* graphs, const uint32_t* const* src,
                                  const uint32_t* const* dst, const double* const* w,
                                  const uint64_t* k, uint32_t count, uint32_t workers,
                                  hl_status* statuses, hl_batch_stats* stats) {
  try {
    need(count == 0 || (graphs && src && dst && k), "NULL argument");
    std::set<const hl_graph*> seen;
    for (uint32_t i = 0; i < count; ++i) {
      need(graphs[i] != nullptr, "graph handle is NULL");
      need(seen.insert(graphs[i]).second, "a graph handle appears twice in one call");
      need(k[i] == 0 || (src[i] && dst[i]), "src/dst are NULL");
    }
  } catch (const std::exception& e) {
    hl_set_error_message(e.what());
    return HL_ERR_INVALID_INPUT;
  }
  if (workers == 0) workers = 16;
  if (workers > count) workers = count;
  std::vector<hl_status> rc(count, HL_OK);
  std::vector<std::string> msg(count);
  // largest batches first, so that the longest graphs do not start last
  std::vector<uint32_t> order(count);
  for (uint32_t i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return k[a] > k[b]; });
  std::atomic<uint32_t> next{0};
  auto run = [&] {
    for (;;) {
      const uint32_t t = next.fetch_add(1);
      if (t >= count) return;
      const uint32_t i = order[t];
      rc[i] = hl::apply_on_handle(graphs[i], src[i], dst[i], w ? w[i] : nullptr, k[i],
                                  stats ? &stats[i] : nullptr, &msg[i]);
    }
  };
  std::vector<std::thread> pool;
  for (uint32_t t = 1; t < workers; ++t) pool.emplace_back(run);
  run();
  for (std::thread& t : pool) t.join();
  hl_status first = HL_OK;
  std::string first_msg;
  for (uint32_t i = 0; i < count; ++i) {
    if (statuses) statuses[i] = rc[i];
    if (rc[i] != HL_OK && first == HL_OK) {
      first = rc[i];
      first_msg = "graph " + std::to_string(i) + ": " + msg[i];
    }
  }
  hl_set_error_message(first_msg);
  return first;
}

HL_API hl_status hl_server_create(uint32_t workers, uint64_t hbm_budget, hl_server** out) {
  HLM_TRY(need(out != nullptr, "out is NULL"); need(workers >= 1 && workers <= 256,
                                                    "workers must be in [1, 256]");
          hl_server* S = new hl_server(); S->budget = hbm_budget;
          for (uint32_t i = 0; i < workers; ++i) S->workers.emplace_back([S] { S->worker_loop(); });
          *out = S);
}

HL_API hl_status hl_server_add_graph(hl_server* S, hl_graph* g, uint32_t* graph_id) {
  HLM_TRY(need(S && g && graph_id, "NULL argument"); std::lock_guard<std::mutex> lk(S->mu);
          for (const GraphSlot& x : S->graphs) need(x.g != g, "graph already registered");
          S->graphs.emplace_back(); S->graphs.back().g = g;
          S->graphs.back().lvl.reset(new LevelCtx());
          S->graphs.back().lvl->server = S;
          S->graphs.back().lvl->graph = (uint32_t)(S->graphs.size() - 1);
          S->graphs.back().bytes = hl::handle_device_bytes(g);
          *graph_id = (uint32_t)(S->graphs.size() - 1));
}

HL_API hl_status hl_server_set_edge_estimate(hl_server* S, uint64_t bytes_per_edge) {
  HLM_TRY(need(S != nullptr, "NULL argument"); std::lock_guard<std::mutex> lk(S->mu);
          S->bytes_per_edge = bytes_per_edge);
}

HL_API hl_status hl_server_set_coalescing(hl_server* S, uint32_t max_requests) {
  HLM_TRY(need(S != nullptr, "NULL argument"); std::lock_guard<std::mutex> lk(S->mu);
          S->max_coalesce = max_requests);
}

HL_API hl_status hl_server_submit(hl_server* S, uint32_t graph_id, const uint32_t* src,
                                  const uint32_t* dst, const double* w, uint64_t k,
                                  uint64_t* request_id) {
  HLM_TRY(need(S != nullptr, "server is NULL"); need(k == 0 || (src && dst), "src/dst are NULL");
          Request r; r.graph = graph_id; r.t_submit = Clock::now();
          r.src.assign(src, src + k); r.dst.assign(dst, dst + k);
          if (w) r.w.assign(w, w + k);
          std::lock_guard<std::mutex> lk(S->mu);
          need(graph_id < S->graphs.size(), "unknown graph id");
          need(!S->stop, "server is shutting down");
          r.id = S->next_id++; r.estimate = S->bytes_per_edge * (k + 1);
          if (request_id) *request_id = r.id;
          ++S->outstanding; S->backlog.push_back(std::move(r)); S->admit_locked());
}

HL_API hl_status hl_server_poll(hl_server* S, hl_request_done* out, uint32_t cap, uint32_t* count,
                                int32_t wait_ms) {
  HLM_TRY(need(S && count, "NULL argument"); need(cap == 0 || out, "out is NULL");
          std::unique_lock<std::mutex> lk(S->mu);
          if (S->done.empty() && wait_ms != 0) {
            auto pred = [&] { return !S->done.empty() || S->outstanding == 0; };
            if (wait_ms < 0) S->cv_done.wait(lk, pred);
            else S->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), pred);
          }
          const uint32_t n = (uint32_t)std::min<size_t>(cap, S->done.size());
          if (n) std::memcpy(out, S->done.data(), n * sizeof(hl_request_done));
          S->done.erase(S->done.begin(), S->done.begin() + n);
          *count = n);
}

HL_API hl_status hl_server_set_level_callback(hl_server* S, hl_server_level_fn fn, void* user) {
  HLM_TRY(need(S != nullptr, "NULL argument"); S->level_user.store(fn ? user : nullptr);
          S->level_fn.store(fn));
}

HL_API hl_status hl_server_drain(hl_server* S) {
  HLM_TRY(need(S != nullptr, "NULL argument"); std::unique_lock<std::mutex> lk(S->mu);
          S->cv_done.wait(lk, [&] { return S->outstanding == 0; }));
}

HL_API void hl_server_destroy(hl_server* S) {
  if (!S) return;
  {
    std::unique_lock<std::mutex> lk(S->mu);
    S->cv_done.wait(lk, [&] { return S->outstanding == 0; });
    S->stop = true;
  }
  S->cv_work.notify_all();
  for (std::thread& t : S->workers) t.join();
  for (GraphSlot& x : S->graphs) hl_set_level_callback(x.g, nullptr, nullptr);
  delete S;
}

}  // extern "C"
