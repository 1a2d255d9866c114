// api.cu — host orchestration (Algorithm 6 level loop, bootstrap) and the
// C ABI declared in include/hl.h and include/hl_debug.h.
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>

#include "../../include/hl_debug.h"
#include "hl_engine.cuh"

using namespace hl;

static thread_local std::string g_err;

void hl_set_error_message(const std::string& m) { g_err = m; }


namespace hl {

u64 Engine::read_u64(const u64* d) {
  if (ktiming) ++kagg[KT_HOST_SYNC].launches;
  HL_CUDA(cudaMemcpyAsync(hs.p, d, sizeof(u64), cudaMemcpyDeviceToHost, stream));
  HL_CUDA(cudaStreamSynchronize(stream));
  return hs.p[0];
}
u32 Engine::read_u32(const u32* d) {
  if (ktiming) ++kagg[KT_HOST_SYNC].launches;
  HL_CUDA(cudaMemcpyAsync(hs.p, d, sizeof(u32), cudaMemcpyDeviceToHost, stream));
  HL_CUDA(cudaStreamSynchronize(stream));
  return (u32)(hs.p[0] & 0xFFFFFFFFull);
}
void Engine::read_u32s(std::initializer_list<const u32*> ptrs, u32* out) {
  if (ktiming) ++kagg[KT_HOST_SYNC].launches;
  require(ptrs.size() <= 16, "too many scalars in one read");
  u32* h = reinterpret_cast<u32*>(hs.p + 32);  // slots 32..39 of the pinned staging
  int i = 0;
  for (const u32* d : ptrs)
    HL_CUDA(cudaMemcpyAsync(h + i++, d, sizeof(u32), cudaMemcpyDeviceToHost, stream));
  HL_CUDA(cudaStreamSynchronize(stream));
  for (int j = 0; j < i; ++j) out[j] = h[j];
}

double Engine::read_f64(const double* d) {
  if (ktiming) ++kagg[KT_HOST_SYNC].launches;
  HL_CUDA(cudaMemcpyAsync(hs.p, d, sizeof(double), cudaMemcpyDeviceToHost, stream));
  HL_CUDA(cudaStreamSynchronize(stream));
  double x;
  std::memcpy(&x, hs.p, sizeof(double));
  return x;
}
void Engine::sync() {
  if (ktiming) ++kagg[KT_HOST_SYNC].launches;
  HL_CUDA(cudaStreamSynchronize(stream));
}

static cudaEvent_t pool_get(std::vector<cudaEvent_t>& pool) {
  if (!pool.empty()) {
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  HL_CUDA(cudaEventCreate(&e));
  return e;
}

cudaEvent_t Engine::kt_begin() {
  if (!ktiming) return nullptr;
  cudaEvent_t e = pool_get(ev_pool);
  HL_CUDA(cudaEventRecord(e, stream));
  return e;
}

void Engine::kt_end(int id, cudaEvent_t a) {
  if (!ktiming || !a) return;
  cudaEvent_t b = pool_get(ev_pool);
  HL_CUDA(cudaEventRecord(b, stream));
  ev_pending.push_back({id, {a, b}});
}

void Engine::kt_collect() {
  if (ev_pending.empty()) return;
  HL_CUDA(cudaStreamSynchronize(stream));
  for (auto& r : ev_pending) {
    float ms = 0.f;
    HL_CUDA(cudaEventElapsedTime(&ms, r.second.first, r.second.second));
    kagg[r.first].ms += ms;
    kagg[r.first].launches += 1;
    ev_pool.push_back(r.second.first);
    ev_pool.push_back(r.second.second);
  }
  ev_pending.clear();
}

}  // namespace hl

namespace {

// Owns the stream; declared first in Holder so it is destroyed last, after
// every stream-ordered free of the engine's buffers.
struct StreamOwner {
  cudaStream_t s = nullptr;
  ~StreamOwner() {
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
};

struct Batchbufs {
  DBuf<u32> u, v;
  DBuf<double> w;
  DBuf<u32> xu[2], xv[2];
  DBuf<double> xw[2];
};

}  // namespace

// The engine plus the buffers that live across calls.
struct EngineBox {
  StreamOwner so;
  std::unique_ptr<Engine> E;
  Batchbufs bb;
};

static void validate_config(const hl_config* c) {
  require(c != nullptr, "config is NULL");
  require(std::isfinite(c->resolution), "resolution must be finite");
  require(c->mode == HL_MODE_DETERMINISTIC || c->mode == HL_MODE_THROUGHPUT,
          "mode must be HL_MODE_DETERMINISTIC or HL_MODE_THROUGHPUT");
  require(c->max_levels >= 1 && c->max_levels <= 64, "max_levels must be in [1, 64]");
}

static void engine_init(EngineBox& B, const hl_config* cfg) {
  validate_config(cfg);
  int ndev = 0;
  HL_CUDA(cudaGetDeviceCount(&ndev));
  require(cfg->device >= 0 && cfg->device < ndev, "device ordinal out of range");
  HL_CUDA(cudaSetDevice(cfg->device));
  HL_CUDA(cudaStreamCreateWithFlags(&B.so.s, cudaStreamNonBlocking));
  B.E.reset(new Engine());
  Engine& E = *B.E;
  E.cfg = *cfg;
  if (!E.cfg.max_rounds) E.cfg.max_rounds = 20;
  E.device = cfg->device;
  E.stream = B.so.s;
  E.mem.stream = B.so.s;
  E.mem.budget = cfg->hbm_budget;
  E.multilevel = cfg->max_levels > 1;
  E.ktiming = (cfg->flags & HL_FLAG_KERNEL_TIMING) != 0;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, cfg->device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  HL_CUDA(cudaEventCreate(&E.ev0));
  HL_CUDA(cudaEventCreate(&E.ev1));
  E.levels.reserve(70);
}

static void engine_free(EngineBox* B) {
  if (!B) return;
  if (B->E) {
    cudaSetDevice(B->E->device);
    if (B->E->ev0) cudaEventDestroy(B->E->ev0);
    if (B->E->ev1) cudaEventDestroy(B->E->ev1);
    B->E->kt_collect();
    for (cudaEvent_t e : B->E->ev_pool) cudaEventDestroy(e);
  }
  delete B;  // members: bb, E (frees on the stream), then so (destroys the stream)
}

namespace hl {

__global__ void k_stats_acc64(const unsigned long long* src, u32 count, unsigned long long* acc) {
  if (threadIdx.x < count) acc[threadIdx.x] += src[threadIdx.x];
}
__global__ void k_stats_acc32(const u32* src, unsigned long long* acc) {
  if (threadIdx.x == 0) *acc += *src;
}
__global__ void k_stats_count_u8(const u8* f, u32 n, unsigned long long* out) {
  u32 local = 0;
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    local += f[i] ? 1u : 0u;
  for (int o = 16; o; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(out, (unsigned long long)local);
}

static void stats_ready(Engine& E) {
  if (E.sc.bacc.cap >= 16) return;
  E.sc.bacc.ensure(E.mem, 16);
  HL_CUDA(cudaMemsetAsync(E.sc.bacc.p, 0, 16 * sizeof(u64), E.stream));
}

void stats_acc_u64(Engine& E, const unsigned long long* src, u32 count, u32 slot) {
  stats_ready(E);
  ++E.nlaunch, k_stats_acc64<<<1, 32, 0, E.stream>>>(
      src, count, reinterpret_cast<unsigned long long*>(E.sc.bacc.p) + slot);
  HL_LAUNCH_CHECK();
}

void stats_acc_u32(Engine& E, const u32* src, u32 slot) {
  stats_ready(E);
  ++E.nlaunch, k_stats_acc32<<<1, 32, 0, E.stream>>>(
      src, reinterpret_cast<unsigned long long*>(E.sc.bacc.p) + slot);
  HL_LAUNCH_CHECK();
}

void stats_count_flags(Engine& E, const u8* flags, u32 n, u32 slot) {
  stats_ready(E);
  if (!n) return;
  u32 g = (n + 255) / 256;
  if (g > 148 * 32) g = 148 * 32;
  ++E.nlaunch, k_stats_count_u8<<<g, 256, 0, E.stream>>>(
      flags, n, reinterpret_cast<unsigned long long*>(E.sc.bacc.p) + slot);
  HL_LAUNCH_CHECK();
}

// A call's statistics start from zero on the device.
static void stats_begin(Engine& E) {
  stats_ready(E);
  HL_CUDA(cudaMemsetAsync(E.sc.bacc.p, 0, 16 * sizeof(u64), E.stream));
  E.sum_nv_batch = 0;
}

}  // namespace hl


// Algorithm 6 (hit_leiden.rs:936-1018) for one batch already on the device.
// NVTX range for the scope (a level, a stage), so that profilers can select
// one level's kernels; a no-op unless a tool is attached.
struct NvtxScope {
  explicit NvtxScope(const char* name) { nvtxRangePushA(name); }
  ~NvtxScope() { nvtxRangePop(); }
  NvtxScope(const NvtxScope&) = delete;
  NvtxScope& operator=(const NvtxScope&) = delete;
};

// Per-level output (hl_set_level_callback): the level's sub-community map is
// copied before its refinement, and the nodes whose entry changed are handed
// to the callback right after it (hit_leiden.rs gives the same point: nothing
// after inc_refinement at level p writes s_cur^p).
__global__ void k_changed_flags(const u32* a, const u32* b, u32 n, u8* flag) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    flag[i] = a[i] != b[i] ? 1 : 0;
}
__global__ void k_gather_u32(const u32* idx, u32 m, const u32* src, u32* out) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < m; i += (u64)gridDim.x * blockDim.x)
    out[i] = src[idx[i]];
}

__global__ void k_flag_ids(const u32* ids, u32 m, u32 n, u8* flags) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < m; i += (u64)gridDim.x * blockDim.x)
    if (ids[i] < n) flags[ids[i]] = 1;
}

static void level_snapshot(Engine& E, Level& L) {
  if (!E.level_fn || !L.g.n) return;
  E.sc.lvl_prev.ensure(E.mem, L.g.n);
  HL_CUDA(cudaMemcpyAsync(E.sc.lvl_prev.p, L.s_cur.p, sizeof(u32) * L.g.n,
                          cudaMemcpyDeviceToDevice, E.stream));
}

static void level_emit(Engine& E, Level& L, u32 p) {
  if (!E.level_fn) return;
  const u32 n = L.g.n;
  std::vector<u32> nodes, ids;
  if (n) {
    Scratch& S = E.sc;
    S.lvl_flag.ensure(E.mem, n);
    S.lvl_nodes.ensure(E.mem, n);
    S.lvl_ids.ensure(E.mem, n);
    S.cnt.ensure(E.mem, 16);
    const u32 g = (u32)std::min<u64>((n + 255) / 256, 148ull * 32);
    ++E.nlaunch, k_changed_flags<<<g, 256, 0, E.stream>>>(S.lvl_prev.p, L.s_cur.p, n, S.lvl_flag.p);
    HL_LAUNCH_CHECK();
    u8* fl = S.lvl_flag.p;
    u32* out = S.lvl_nodes.p;
    u32* cnt = S.cnt.p + 14;
    cub_run(E, [&](void* t, size_t& b) {
      return cub::DeviceSelect::Flagged(t, b, cub::CountingInputIterator<u32>(0), fl, out, cnt,
                                        (int64_t)n, E.stream);
    });
    const u32 m = E.read_u32(cnt);
    if (m) {
      ++E.nlaunch, k_gather_u32<<<(u32)std::min<u64>((m + 255) / 256, 148ull * 32), 256, 0,
                                   E.stream>>>(out, m, L.s_cur.p, S.lvl_ids.p);
      HL_LAUNCH_CHECK();
      nodes.resize(m);
      ids.resize(m);
      HL_CUDA(cudaMemcpyAsync(nodes.data(), out, sizeof(u32) * m, cudaMemcpyDeviceToHost,
                              E.stream));
      HL_CUDA(cudaMemcpyAsync(ids.data(), S.lvl_ids.p, sizeof(u32) * m, cudaMemcpyDeviceToHost,
                              E.stream));
      E.sync();
    }
  }
  E.level_fn(E.level_user, p, (uint64_t)nodes.size(), nodes.data(), ids.data());
}

static void hit_leiden_batch(EngineBox& B, const DevEdges& delta) {
  Engine& E = *B.E;
  hl_batch_stats& st = E.st;
  const u32 P = (u32)E.levels.size();
  if (!E.multilevel) {
    // The reference's reachable configuration: one level (state.rs:42), so
    // no aggregation, and def_update is a no-op (hit_leiden.rs:1773-1792).
    Level& L = E.levels[0];
    apply_delta(E, L, delta, L.g.n, (E.cfg.flags & HL_FLAG_KEEP_SELF_LOOPS) != 0);
    MoveOut mo = inc_movement(E, L, delta, delta.k == 0, false);
    stats_count_flags(E, E.sc.changed.p, L.g.n, 10);
    level_snapshot(E, L);
    RefineOut ro = inc_refinement(E, L, false);
    level_emit(E, L, 0);
    st.iterations += mo.iterations;
    st.moves += mo.moves;
    st.candidates += mo.candidates;
    st.traversed += mo.traversed;
    st.splits += ro.splits;
    st.merges += ro.merges;
    st.refined = ro.refined;
    return;
  }
  DevEdges cur = delta;
  u32 cur_n = E.levels[0].g.n;
  E.k_flags_set = false;
  for (u32 p = 0; p < P; ++p) {
    char level_name[24];
    std::snprintf(level_name, sizeof(level_name), "level%u", p);
    NvtxScope level_range(level_name);
    Level& L = E.levels[p];
    cudaEvent_t e0 = E.kt_begin();
    {
      NvtxScope r("apply");
      apply_delta(E, L, cur, cur_n > L.g.n ? cur_n : L.g.n, true);
    }
    E.kt_end(KT_STAGE_APPLY, e0);
    e0 = E.kt_begin();
    MoveOut mo;
    {
      NvtxScope r("move");
      mo = inc_movement(E, L, cur, cur.k == 0, true);
    }
    E.kt_end(KT_STAGE_MOVE, e0);
    if (p == 0) stats_count_flags(E, E.sc.changed.p, L.g.n, 10);
    e0 = E.kt_begin();
    RefineOut ro;
    level_snapshot(E, L);
    {
      NvtxScope r("refine");
      ro = inc_refinement(E, L, true);
    }
    E.kt_end(KT_STAGE_REFINE, e0);
    level_emit(E, L, p);
    st.iterations += mo.iterations;
    st.moves += mo.moves;
    st.candidates += mo.candidates;
    st.traversed += mo.traversed;
    st.splits += ro.splits;
    st.merges += ro.merges;
    if (p == 0) st.refined = ro.refined;
    if (p + 1 >= P) break;
    Level& H = E.levels[p + 1];
    // Grow level p+1 to hold every sub-community id handed out at level p.
    u32 need = 0;
    {
      u32* o = E.sc.cnt.p + 12;
      u32* sc = L.s_cur.p;
      cub_run(E, [&](void* t, size_t& b) {
        return cub::DeviceReduce::Max(t, b, sc, o, (int64_t)L.g.n, E.stream);
      });
      need = E.read_u32(o) + 1;
      for (auto& xo : E.new_ids) need = need > xo.first + 1 ? need : xo.first + 1;
    }
    graph_grow_nodes(E, H, need);
    inherit_new_nodes(E, H, E.new_ids);
    // M8: the nodes level p+1 gains from this level's splits, and those whose
    // community the projection changes, join K at level p+1
    E.sc.kflag.ensure(E.mem, H.g.n ? H.g.n : 1);
    HL_CUDA(cudaMemsetAsync(E.sc.kflag.p, 0, H.g.n ? H.g.n : 1, E.stream));
    if (!E.new_ids.empty()) {
      std::vector<u32> ids;
      for (auto& xo : E.new_ids) ids.push_back(xo.first);
      E.sc.kflag_ids.ensure(E.mem, ids.size());
      HL_CUDA(cudaMemcpyAsync(E.sc.kflag_ids.p, ids.data(), sizeof(u32) * ids.size(),
                              cudaMemcpyHostToDevice, E.stream));
      ++E.nlaunch, k_flag_ids<<<(u32)std::min<size_t>((ids.size() + 255) / 256, 148 * 32), 256, 0,
                                E.stream>>>(E.sc.kflag_ids.p, (u32)ids.size(), H.g.n,
                                            E.sc.kflag.p);
      HL_LAUNCH_CHECK();
    }
    project_up(E, L, H, E.sc.kflag.p);
    E.k_flags_set = true;
    if (cur.k == 0 && ro.refined == 0) {  // should_skip_aggregation (:1020-1022)
      cur = DevEdges{};
      cur_n = H.g.n;
      continue;
    }
    u32 nn = 0;
    e0 = E.kt_begin();
    u64 cnt;
    {
      NvtxScope r("aggregate");
      cnt = inc_aggregation(E, L, cur, &nn, true, true);
    }
    E.kt_end(KT_STAGE_AGGREGATE, e0);
    int slot = (p + 1) & 1;
    B.bb.xu[slot].ensure(E.mem, cnt ? cnt : 1);
    B.bb.xv[slot].ensure(E.mem, cnt ? cnt : 1);
    B.bb.xw[slot].ensure(E.mem, cnt ? cnt : 1);
    if (cnt) {
      HL_CUDA(cudaMemcpyAsync(B.bb.xu[slot].p, E.sc.eu2.p, sizeof(u32) * cnt,
                              cudaMemcpyDeviceToDevice, E.stream));
      HL_CUDA(cudaMemcpyAsync(B.bb.xv[slot].p, E.sc.ev2.p, sizeof(u32) * cnt,
                              cudaMemcpyDeviceToDevice, E.stream));
      HL_CUDA(cudaMemcpyAsync(B.bb.xw[slot].p, E.sc.ew2.p, sizeof(double) * cnt,
                              cudaMemcpyDeviceToDevice, E.stream));
    }
    cur = DevEdges{B.bb.xu[slot].p, B.bb.xv[slot].p, B.bb.xw[slot].p, cnt};
    cur_n = nn > H.g.n ? nn : H.g.n;
  }
  top_down(E);
}

// Multi-level bootstrap (the spec's Algorithm 1): Move, Refine, Aggregate per
// level until a level no longer coarsens by 1% or max_levels is reached.
static void bootstrap(EngineBox& B, u32 n, const DevEdges& G) {
  Engine& E = *B.E;
  E.levels.clear();
  E.levels.emplace_back();
  graph_init_empty(E, E.levels[0], n);
  if (!E.multilevel) {
    // PartitionState::identity + an empty supergraph + hit_leiden(G): the
    // reference tests' bootstrap (hit_leiden.rs:3119-3126).
    hit_leiden_batch(B, G);
    return;
  }
  apply_delta(E, E.levels[0], G, n, true);
  u32 p = 0;
  while (true) {
    Level& L = E.levels[p];
    const u32 np = L.g.n;
    MoveOut mo = inc_movement(E, L, DevEdges{}, true, true);
    RefineOut ro = inc_refinement(E, L, true);
    E.st.iterations += mo.iterations;
    E.st.moves += mo.moves;
    E.st.traversed += mo.traversed;
    E.st.merges += ro.merges;
    u32 smax = 0;
    {
      u32* o = E.sc.cnt.p + 12;
      u32* sc = L.s_cur.p;
      cub_run(E, [&](void* t, size_t& b) {
        return cub::DeviceReduce::Max(t, b, sc, o, (int64_t)np, E.stream);
      });
      smax = E.read_u32(o);
    }
    u32 nn = np ? rank_compact(E, L.s_cur.p, np, smax) : 0;
    if (np)
      HL_CUDA(cudaMemcpyAsync(L.s_pre.p, L.s_cur.p, sizeof(u32) * np, cudaMemcpyDeviceToDevice,
                              E.stream));
    if (p + 1 >= E.cfg.max_levels || nn <= 1 || (u64)nn * 100 >= (u64)np * 99) break;
    u64 cnt = aggregate_full(E, L, L.s_cur.p, nullptr, nullptr, nullptr);
    E.levels.emplace_back();
    Level& H = E.levels[p + 1];
    Level& Lr = E.levels[p];
    graph_init_empty(E, H, nn);
    apply_delta(E, H, DevEdges{E.sc.eu2.p, E.sc.ev2.p, E.sc.ew2.p, cnt}, nn, true);
    project_up(E, Lr, H);
    ++p;
  }
  top_down(E);
}

#define HL_TRY(...)                                            \
  try {                                                        \
    __VA_ARGS__;                                               \
    g_err.clear();                                             \
    return HL_OK;                                              \
  } catch (const hl::Error& e) {                               \
    g_err = e.what();                                          \
    return e.status;                                           \
  } catch (const std::exception& e) {                          \
    g_err = e.what();                                          \
    return HL_ERR_CUDA;                                        \
  } catch (...) {                                              \
    g_err = "unknown error";                                   \
    return HL_ERR_CUDA;                                        \
  }

static EngineBox* box(hl_graph* g) { return reinterpret_cast<EngineBox*>(g); }
static const EngineBox* box(const hl_graph* g) { return reinterpret_cast<const EngineBox*>(g); }

static void upload_edges(EngineBox& B, const uint32_t* src, const uint32_t* dst, const double* w,
                         uint64_t m, DevEdges& out) {
  Engine& E = *B.E;
  B.bb.u.ensure(E.mem, m ? m : 1);
  B.bb.v.ensure(E.mem, m ? m : 1);
  if (m) {
    HL_CUDA(cudaMemcpyAsync(B.bb.u.p, src, sizeof(u32) * m, cudaMemcpyHostToDevice, E.stream));
    HL_CUDA(cudaMemcpyAsync(B.bb.v.p, dst, sizeof(u32) * m, cudaMemcpyHostToDevice, E.stream));
  }
  const double* dw = nullptr;
  if (w && m) {
    B.bb.w.ensure(E.mem, m);
    HL_CUDA(cudaMemcpyAsync(B.bb.w.p, w, sizeof(double) * m, cudaMemcpyHostToDevice, E.stream));
    dw = B.bb.w.p;
  }
  out = DevEdges{B.bb.u.p, B.bb.v.p, dw, m};
}

static void finish_stats(EngineBox& B, hl_batch_stats* stats) {
  Engine& E = *B.E;
  // the statistics kept on the device come back with the call's last wait
  stats_ready(E);
  HL_CUDA(cudaMemcpyAsync(E.hs.p + 40, E.sc.bacc.p, 16 * sizeof(u64), cudaMemcpyDeviceToHost,
                          E.stream));
  HL_CUDA(cudaEventRecord(E.ev1, E.stream));
  HL_CUDA(cudaEventSynchronize(E.ev1));
  float ms = 0.f;
  HL_CUDA(cudaEventElapsedTime(&ms, E.ev0, E.ev1));
  E.st.device_ms = ms;
  E.st.launches = E.nlaunch - E.launch_mark;
  u64 acc[16];
  std::memcpy(acc, E.hs.p + 40, sizeof(acc));
  u64 trav = 0, ncand = 0;
  const int bins[4] = {KT_EVAL_SMALL, KT_EVAL_MID, KT_EVAL_BIG, KT_EVAL_HUGE};
  for (int b = 0; b < 4; ++b) {
    trav += acc[2 * b];
    ncand += acc[2 * b + 1];
    E.kagg[bins[b]].bytes += 16ull * acc[2 * b] + 8ull * acc[2 * b + 1];
  }
  // Algorithmic bytes of the evaluation: per active vertex its list entry,
  // offsets, f, k, d(f) and outputs; per adjacency entry the neighbour,
  // weight and neighbour community; per evaluated candidate its d(C).
  E.kagg[KT_MOVE_EVAL].bytes += 52ull * E.sum_nv_batch + 16ull * trav + 8ull * ncand;
  E.st.traversed += trav;
  E.st.moves += acc[8];
  E.st.merges += acc[9];
  E.st.changed = acc[10];
  E.kt_collect();
  E.st.levels = (u32)E.levels.size();
  E.st.edges = E.levels.empty() ? 0 : E.levels[0].g.nnz / 2;
  E.st.modularity = NAN;
  if (E.cfg.flags & HL_FLAG_BATCH_MODULARITY)
    E.st.modularity = modularity(E, E.levels[0], E.levels[0].f.p);
  if (stats) *stats = E.st;
}

static void create_impl(const hl_config* cfg, uint32_t n, const uint32_t* src, const uint32_t* dst,
                        const double* w, uint64_t m, bool device_ptrs, hl_graph** out) {
  require(out != nullptr, "out is NULL");
  require(m == 0 || (src && dst), "src/dst are NULL");
  std::unique_ptr<EngineBox> B(new EngineBox());
  engine_init(*B, cfg);
  Engine& E = *B->E;
  DevEdges G;
  if (device_ptrs)
    G = DevEdges{src, dst, w, m};
  else
    upload_edges(*B, src, dst, w, m, G);
  check_endpoints(E, G, n);
  E.integral = edges_integral(E, G);
  E.st = hl_batch_stats{};
  stats_begin(E);
  HL_CUDA(cudaEventRecord(E.ev0, E.stream));
  E.in_bootstrap = true;
  bootstrap(*B, n, G);
  E.in_bootstrap = false;
  if (E.levels[0].tw >= 4503599627370496.0) E.integral = false;  // 2^52
  finish_stats(*B, nullptr);
  // The bootstrap's scratch (sorts over the whole edge list) is far larger
  // than an update batch needs: hand it back; batches regrow what they use.
  E.sc = Scratch();
  E.sync();
  *out = reinterpret_cast<hl_graph*>(B.release());
}

static void apply_impl(hl_graph* g, const uint32_t* src, const uint32_t* dst, const double* w,
                       uint64_t k, bool device_ptrs, hl_batch_stats* stats) {
  require(g != nullptr, "graph handle is NULL");
  require(k == 0 || (src && dst), "src/dst are NULL");
  EngineBox& B = *box(g);
  Engine& E = *B.E;
  HL_CUDA(cudaSetDevice(E.device));
  E.st = hl_batch_stats{};
  stats_begin(E);
  E.launch_mark = E.nlaunch;
  DevEdges D;
  if (device_ptrs)
    D = DevEdges{src, dst, w, k};
  else
    upload_edges(B, src, dst, w, k, D);
  // device_ms starts with the batch resident on the device: the host→device
  // copy of a host batch is not part of it.
  HL_CUDA(cudaEventRecord(E.ev0, E.stream));
  check_endpoints(E, D, E.levels[0].g.n);
  if (E.integral && !edges_integral(E, D)) E.integral = false;
  hit_leiden_batch(B, D);
  if (E.levels[0].tw >= 4503599627370496.0) E.integral = false;
  finish_stats(B, stats);
}

namespace hl {

// Entry points for the multi-graph executors (multi.cu): one batch on one
// handle, with the error captured for the calling thread; device bytes held.
hl_status apply_on_handle(hl_graph* g, const uint32_t* src, const uint32_t* dst, const double* w,
                          uint64_t k, hl_batch_stats* stats, std::string* err) {
  try {
    apply_impl(g, src, dst, w, k, false, stats);
    return HL_OK;
  } catch (const Error& e) {
    if (err) *err = e.what();
    return e.status;
  } catch (const std::exception& e) {
    if (err) *err = e.what();
    return HL_ERR_CUDA;
  } catch (...) {
    if (err) *err = "unknown error";
    return HL_ERR_CUDA;
  }
}

u64 handle_device_bytes(const hl_graph* g) { return box(g)->E->mem.used; }

}  // namespace hl

extern "C" {

hl_status hl_config_default(hl_config* cfg) {
  if (!cfg) {
    g_err = "config is NULL";
    return HL_ERR_INVALID_INPUT;
  }
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->resolution = 1.0;
  cfg->mode = HL_MODE_DETERMINISTIC;  // RunConfig::default() (config.rs:40-43)
  cfg->max_levels = 10;
  cfg->max_rounds = 20;
  cfg->flags = 0;
  cfg->hbm_budget = 0;
  cfg->device = 0;
  return HL_OK;
}

hl_status hl_create(const hl_config* cfg, uint32_t n, const uint32_t* src, const uint32_t* dst,
                    const double* w, uint64_t m, hl_graph** out) {
  HL_TRY(create_impl(cfg, n, src, dst, w, m, false, out));
}

hl_status hl_create_device(const hl_config* cfg, uint32_t n, const uint32_t* src,
                           const uint32_t* dst, const double* w, uint64_t m, hl_graph** out) {
  HL_TRY(create_impl(cfg, n, src, dst, w, m, true, out));
}

hl_status hl_apply_batch(hl_graph* g, const uint32_t* src, const uint32_t* dst, const double* w,
                         uint64_t k, hl_batch_stats* stats) {
  HL_TRY(apply_impl(g, src, dst, w, k, false, stats));
}

hl_status hl_apply_batch_device(hl_graph* g, const uint32_t* src, const uint32_t* dst,
                                const double* w, uint64_t k, hl_batch_stats* stats) {
  HL_TRY(apply_impl(g, src, dst, w, k, true, stats));
}

static const char* kernel_names[KT_COUNT] = {
    "move_eval",   "refine_eval", "select_decoupled", "csr_merge_rows", "aggregate_compress",
    "eval_small",  "eval_mid",    "eval_wide",        "eval_huge",      "comm_degrees",
    "apply_and_mark",
    "refine_cc",   "t_filter",    "row_sums",         "delta_resolve",  "stage_apply",
    "stage_move",  "stage_refine", "stage_aggregate", "host_syncs",
    "csr_copy_untouched", "move_small_rounds", "eval_huge_partitioned"};

hl_status hl_kernel_stats(const hl_graph* g, hl_kernel_stat* out, uint32_t cap, uint32_t* count) {
  HL_TRY(require(g && count, "NULL argument"); Engine& E = *const_cast<EngineBox*>(box(g))->E;
         E.kt_collect(); *count = KT_COUNT; for (uint32_t i = 0; i < KT_COUNT && i < cap && out; ++i) {
           std::memset(&out[i], 0, sizeof(out[i]));
           std::strncpy(out[i].name, kernel_names[i], sizeof(out[i].name) - 1);
           out[i].launches = E.kagg[i].launches;
           out[i].total_ms = E.kagg[i].ms;
           out[i].bytes = E.kagg[i].bytes;
           out[i].items = E.kagg[i].items;
         });
}

hl_status hl_reset_kernel_stats(hl_graph* g) {
  HL_TRY(require(g != nullptr, "NULL argument"); Engine& E = *box(g)->E; E.kt_collect();
         for (auto& k : E.kagg) k = KernelAgg{});
}

hl_status hl_set_resolution(hl_graph* g, double gamma) {
  HL_TRY(require(g != nullptr, "graph handle is NULL");
         require(std::isfinite(gamma), "resolution must be finite");
         box(g)->E->cfg.resolution = gamma);
}

hl_status hl_set_level_callback(hl_graph* g, hl_level_fn fn, void* user) {
  HL_TRY(require(g != nullptr, "graph handle is NULL"); box(g)->E->level_fn = fn;
         box(g)->E->level_user = fn ? user : nullptr);
}

hl_status hl_autotune_info(const hl_graph* g, uint32_t* mid_max, uint32_t* wide_max,
                           uint32_t* hub_defer, uint32_t* frontier) {
  HL_TRY(require(g && mid_max && wide_max && frontier, "NULL argument");
         const Engine& E = *box(g)->E; *mid_max = E.tune.mid_max ? E.tune.mid_max : 128;
         *wide_max = E.tune.wide_max ? E.tune.wide_max : 512;
         if (hub_defer) *hub_defer = E.tune.hub_defer ? E.tune.hub_defer : 8192;
         *frontier = E.tune.done ? E.tune.frontier : 0);
}

hl_status hl_set_mode(hl_graph* g, uint32_t mode) {
  HL_TRY(require(g != nullptr, "graph handle is NULL");
         require(mode == HL_MODE_DETERMINISTIC || mode == HL_MODE_THROUGHPUT,
                 "mode must be HL_MODE_DETERMINISTIC or HL_MODE_THROUGHPUT");
         box(g)->E->cfg.mode = mode);
}

hl_status hl_num_nodes(const hl_graph* g, uint32_t* n) {
  HL_TRY(require(g && n, "NULL argument"); *n = box(g)->E->levels[0].g.n);
}

hl_status hl_num_levels(const hl_graph* g, uint32_t* levels) {
  HL_TRY(require(g && levels, "NULL argument"); *levels = (uint32_t)box(g)->E->levels.size());
}

hl_status hl_level_size(const hl_graph* g, uint32_t level, uint32_t* n_level) {
  HL_TRY(require(g && n_level, "NULL argument");
         require(level < box(g)->E->levels.size(), "level out of range");
         *n_level = box(g)->E->levels[level].g.n);
}

hl_status hl_num_edges(const hl_graph* g, uint32_t level, uint64_t* entries) {
  HL_TRY(require(g && entries, "NULL argument");
         require(level < box(g)->E->levels.size(), "level out of range");
         *entries = box(g)->E->levels[level].g.nnz);
}

static void get_map_impl(const hl_graph* g, uint32_t level, uint32_t which, uint32_t* out) {
  require(g && out, "NULL argument");
  Engine& E = *const_cast<EngineBox*>(box(g))->E;
  require(level < E.levels.size(), "level out of range");
  HL_CUDA(cudaSetDevice(E.device));
  Level& L = E.levels[level];
  const u32* src = nullptr;
  switch (which) {
    case HL_MAP_COMMUNITY: src = L.f.p; break;
    case HL_MAP_REFINED: src = L.gm.p; break;
    case HL_MAP_SUB_PREVIOUS: src = L.s_pre.p; break;
    case HL_MAP_SUB_CURRENT: src = L.s_cur.p; break;
    default: require(false, "unknown map");
  }
  if (L.g.n)
    HL_CUDA(cudaMemcpyAsync(out, src, sizeof(u32) * L.g.n, cudaMemcpyDeviceToHost, E.stream));
  E.sync();
}

hl_status hl_get_map(const hl_graph* g, uint32_t level, uint32_t which, uint32_t* out) {
  HL_TRY(get_map_impl(g, level, which, out));
}

static void get_partition_impl(const hl_graph* g, uint32_t* out) {
  require(g && out, "NULL argument");
  Engine& E = *const_cast<EngineBox*>(box(g))->E;
  HL_CUDA(cudaSetDevice(E.device));
  Level& L = E.levels[0];
  u32 n = L.g.n;
  if (!n) return;
  DBuf<u32> tmp;
  tmp.ensure(E.mem, n);
  canonicalize_device(E, L.f.p, n, tmp.p);
  HL_CUDA(cudaMemcpyAsync(out, tmp.p, sizeof(u32) * n, cudaMemcpyDeviceToHost, E.stream));
  E.sync();
}

hl_status hl_get_partition(const hl_graph* g, uint32_t* out) { HL_TRY(get_partition_impl(g, out)); }

static void get_csr_impl(const hl_graph* g, uint32_t level, uint64_t* off, uint32_t* col,
                         double* w) {
  require(g != nullptr, "NULL argument");
  Engine& E = *const_cast<EngineBox*>(box(g))->E;
  require(level < E.levels.size(), "level out of range");
  HL_CUDA(cudaSetDevice(E.device));
  DevGraph& G = E.levels[level].g;
  if (off)
    HL_CUDA(cudaMemcpyAsync(off, G.off.p, sizeof(u64) * ((size_t)G.n + 1), cudaMemcpyDeviceToHost,
                            E.stream));
  if (col && G.nnz)
    HL_CUDA(cudaMemcpyAsync(col, G.col.p, sizeof(u32) * G.nnz, cudaMemcpyDeviceToHost, E.stream));
  if (w && G.nnz)
    HL_CUDA(cudaMemcpyAsync(w, G.w.p, sizeof(double) * G.nnz, cudaMemcpyDeviceToHost, E.stream));
  E.sync();
}

hl_status hl_get_csr(const hl_graph* g, uint32_t level, uint64_t* off, uint32_t* col, double* w) {
  HL_TRY(get_csr_impl(g, level, off, col, w));
}

static void modularity_impl(const hl_graph* g, const uint32_t* part, double* q) {
  require(g && q, "NULL argument");
  Engine& E = *const_cast<EngineBox*>(box(g))->E;
  HL_CUDA(cudaSetDevice(E.device));
  Level& L = E.levels[0];
  if (!part) {
    *q = modularity(E, L, L.f.p);
    return;
  }
  DBuf<u32> tmp;
  tmp.ensure(E.mem, L.g.n ? L.g.n : 1);
  if (L.g.n)
    HL_CUDA(cudaMemcpyAsync(tmp.p, part, sizeof(u32) * L.g.n, cudaMemcpyHostToDevice, E.stream));
  *q = modularity(E, L, tmp.p);
}

hl_status hl_modularity(const hl_graph* g, double* q) { HL_TRY(modularity_impl(g, nullptr, q)); }

hl_status hl_modularity_of(const hl_graph* g, const uint32_t* part, double* q) {
  HL_TRY(require(part != nullptr, "part is NULL"); modularity_impl(g, part, q));
}

hl_status hl_device_bytes(const hl_graph* g, uint64_t* used, uint64_t* peak) {
  HL_TRY(require(g != nullptr, "graph handle is NULL"); const Engine& E = *box(g)->E;
         if (used) *used = E.mem.used; if (peak) *peak = E.mem.peak);
}

void hl_destroy(hl_graph* g) {
  try {
    engine_free(box(g));
  } catch (...) {
  }
}

const char* hl_last_error(void) { return g_err.c_str(); }

const char* hl_version(void) { return "hit-leiden-b200 0.1.0 (sm_100a)"; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Function-level entry points (include/hl_debug.h)
// ---------------------------------------------------------------------------
namespace {

// RunMode of the stage entry points (hl_dbg_set_mode); Throughput unless set.
std::atomic<uint32_t> g_dbg_mode{HL_MODE_THROUGHPUT};
// Degree-bin thresholds of the stage entry points (hl_dbg_set_bins).
std::atomic<uint32_t> g_dbg_mid{0}, g_dbg_wide{0};

std::unique_ptr<EngineBox> scratch_engine(int32_t device) {
  hl_config cfg;
  hl_config_default(&cfg);
  cfg.device = device;
  cfg.mode = g_dbg_mode.load();
  std::unique_ptr<EngineBox> B(new EngineBox());
  engine_init(*B, &cfg);
  B->E->tune.mid_max = g_dbg_mid.load();
  B->E->tune.wide_max = g_dbg_wide.load();
  B->E->tune.done = true;
  return B;
}

bool host_integral(const double* w, u64 n) {
  if (!w) return true;
  for (u64 i = 0; i < n; ++i)
    if (!(w[i] == std::floor(w[i])) || std::fabs(w[i]) > 4294967296.0) return false;
  return true;
}

template <typename T>
void up(Engine& E, DBuf<T>& b, const T* h, size_t n) {
  b.ensure(E.mem, n ? n : 1);
  if (n && h) HL_CUDA(cudaMemcpyAsync(b.p, h, sizeof(T) * n, cudaMemcpyHostToDevice, E.stream));
}

template <typename T>
void down(Engine& E, T* h, const T* d, size_t n) {
  if (n && h) HL_CUDA(cudaMemcpyAsync(h, d, sizeof(T) * n, cudaMemcpyDeviceToHost, E.stream));
}

void level_from_host(Engine& E, Level& L, u32 n, const u64* off, const u32* col, const double* w) {
  graph_init_empty(E, L, n);
  u64 nnz = off ? off[n] : 0;
  L.g.nnz = nnz;
  up(E, L.g.off, off, (size_t)n + 1);
  up(E, L.g.col, col, nnz);
  up(E, L.g.w, w, nnz);
  u64 loops = 0;
  for (u32 v = 0; v < n; ++v)
    for (u64 p = off[v]; p < off[v + 1]; ++p)
      if (col[p] == v) ++loops;
  L.g.self_loop_entries = loops;
  E.integral = host_integral(w, nnz);
  recompute_all_degrees(E, L);
}

DevEdges edges_up(Engine& E, Batchbufs& bb, const u32* s, const u32* d, const double* w, u64 k) {
  up(E, bb.u, s, k);
  up(E, bb.v, d, k);
  const double* dw = nullptr;
  if (w && k) {
    up(E, bb.w, w, k);
    dw = bb.w.p;
  }
  return DevEdges{bb.u.p, bb.v.p, dw, k};
}

}  // namespace

extern "C" {

hl_status hl_dbg_tree_sum(int32_t device, const double* x, uint64_t n, double* out) {
  HL_TRY({
    auto B = scratch_engine(device);
    Engine& E = *B->E;
    DBuf<double> d;
    up(E, d, x, n);
    *out = tree_sum(E, d.p, n);
  });
}

hl_status hl_dbg_seq_sums(int32_t device, uint32_t nseg, const uint64_t* off, const double* x,
                          double init, int32_t path, double* out) {
  HL_TRY({
    require(nseg == 0 || (off && x && out), "NULL argument");
    require(path >= 0 && path <= 2, "path must be 0, 1 or 2");
    auto B = scratch_engine(device);
    Engine& E = *B->E;
    if (nseg) {
      const u64 total = off[nseg];
      for (u32 i = 0; i < nseg; ++i) require(off[i] <= off[i + 1], "offsets must ascend");
      DBuf<u64> doff;
      DBuf<double> dx, dout;
      up(E, doff, off, (size_t)nseg + 1);
      up(E, dx, x, total);
      dout.ensure(E.mem, nseg);
      seq_sums(E, nseg, doff.p, dx.p, init, path, dout.p);
      down(E, out, dout.p, nseg);
      E.sync();
    }
  });
}

hl_status hl_dbg_move_eval(int32_t device, uint32_t n, const uint64_t* off, const uint32_t* col,
                           const double* w, const uint32_t* f, const double* d, uint64_t d_len,
                           const double* k, double tw, double gamma, const uint32_t* verts,
                           uint64_t nv, uint32_t* out_to, double* out_gain) {
  HL_TRY({
    auto B = scratch_engine(device);
    Engine& E = *B->E;
    E.cfg.resolution = gamma;
    Level L;
    level_from_host(E, L, n, off, col, w);
    up(E, L.f, f, n);
    up(E, L.k, k, n);
    L.tw = tw;
    DBuf<double> dd;
    up(E, dd, d, d_len);
    DBuf<u32> vv, to;
    DBuf<double> g;
    up(E, vv, verts, nv);
    to.ensure(E.mem, nv ? nv : 1);
    g.ensure(E.mem, nv ? nv : 1);
    run_eval(E, 0, vv.p, (u32)nv, L, L.s_cur.p, dd.p, nullptr, true, to.p, g.p, nullptr);
    down(E, out_to, to.p, nv);
    down(E, out_gain, g.p, nv);
    E.sync();
  });
}

hl_status hl_dbg_select_decoupled(int32_t device, const uint32_t* node, const uint32_t* from,
                                  const uint32_t* to, const double* gain, uint64_t m,
                                  uint32_t* out_nodes, uint64_t* out_count) {
  HL_TRY({
    auto B = scratch_engine(device);
    Engine& E = *B->E;
    // Rank order: gain descending, node ascending (throughput.rs:205-210).
    std::vector<u64> order(m);
    for (u64 i = 0; i < m; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](u64 a, u64 b) { return node[a] < node[b]; });
    std::vector<u32> sn, sf, stt;
    std::vector<double> sg;
    for (u64 i : order)
      if (gain[i] > 0.0) {
        sn.push_back(node[i]);
        sf.push_back(from[i]);
        stt.push_back(to[i]);
        sg.push_back(gain[i]);
      }
    std::vector<u64> rk(sn.size());
    for (u64 i = 0; i < rk.size(); ++i) rk[i] = i;
    std::stable_sort(rk.begin(), rk.end(), [&](u64 a, u64 b) { return sg[a] > sg[b]; });
    u32 M = (u32)rk.size();
    std::vector<u32> rf(M), rt(M), rn(M);
    u32 mx = 0;
    for (u32 r = 0; r < M; ++r) {
      rf[r] = sf[rk[r]];
      rt[r] = stt[rk[r]];
      rn[r] = sn[rk[r]];
      mx = std::max(mx, std::max(rf[r], rt[r]));
    }
    Scratch& S = E.sc;
    S.cnt.ensure(E.mem, 16);
    ensure_comm_arrays(E, (size_t)mx + 2);
    up(E, S.sel_from, rf.data(), M);
    up(E, S.sel_to, rt.data(), M);
    S.status.ensure(E.mem, M ? M : 1);
    S.nmask.ensure(E.mem, M ? M : 1);
    u64 cntv = 0;
    if (M) {
      select_decoupled_dev(E, M);
      std::vector<u8> stv(M);
      down(E, stv.data(), S.status.p, M);
      E.sync();
      for (u32 r = 0; r < M; ++r)
        if (stv[r] == 1) out_nodes[cntv++] = rn[r];
    }
    *out_count = cntv;
  });
}

hl_status hl_dbg_apply_delta(int32_t device, uint32_t n, const uint64_t* off, const uint32_t* col,
                             const double* w, uint32_t delta_n, const uint32_t* dsrc,
                             const uint32_t* ddst, const double* dw, uint64_t dk,
                             int32_t keep_self_loops, uint64_t* out_off, uint32_t* out_col,
                             double* out_w, uint64_t cap, uint64_t* out_nnz) {
  HL_TRY({
    auto B = scratch_engine(device);
    Engine& E = *B->E;
    Level L;
    level_from_host(E, L, n, off, col, w);
    DevEdges D = edges_up(E, B->bb, dsrc, ddst, dw, dk);
    if (!host_integral(dw, dk)) E.integral = false;
    u32 nn = std::max(n, delta_n);
    check_endpoints(E, D, nn);
    apply_delta(E, L, D, nn, keep_self_loops != 0);
    *out_nnz = L.g.nnz;
    require(L.g.nnz <= cap, "output capacity too small");
    down(E, out_off, L.g.off.p, (size_t)L.g.n + 1);
    down(E, out_col, L.g.col.p, L.g.nnz);
    down(E, out_w, L.g.w.p, L.g.nnz);
    E.sync();
  });
}

hl_status hl_dbg_inc_movement(int32_t device, uint32_t n, const uint64_t* off, const uint32_t* col,
                              const double* w, const uint32_t* dsrc, const uint32_t* ddst,
                              const double* dw, uint64_t dk, uint32_t* f, const uint32_t* s,
                              double gamma, uint32_t max_rounds, int32_t mark_moved,
                              uint8_t* changed, uint8_t* affected, uint32_t* iterations) {
  HL_TRY({
    auto B = scratch_engine(device);
    Engine& E = *B->E;
    E.cfg.resolution = gamma;
    E.cfg.max_rounds = max_rounds ? max_rounds : 20;
    Level L;
    level_from_host(E, L, n, off, col, w);
    up(E, L.f, f, n);
    up(E, L.s_cur, s, n);
    DevEdges D = edges_up(E, B->bb, dsrc, ddst, dw, dk);
    MoveOut mo = inc_movement(E, L, D, dk == 0, mark_moved != 0);
    down(E, f, L.f.p, n);
    down(E, changed, E.sc.changed.p, n);
    down(E, affected, E.sc.affected.p, n);
    E.sync();
    if (iterations) *iterations = mo.iterations;
  });
}

hl_status hl_dbg_inc_refinement(int32_t device, uint32_t n, const uint64_t* off,
                                const uint32_t* col, const double* w, const uint32_t* f,
                                uint32_t* s, const uint8_t* affected, double gamma,
                                int32_t cc_same_community, uint8_t* refined) {
  HL_TRY({
    auto B = scratch_engine(device);
    Engine& E = *B->E;
    E.cfg.resolution = gamma;
    Level L;
    level_from_host(E, L, n, off, col, w);
    up(E, L.f, f, n);
    up(E, L.s_cur, s, n);
    up(E, E.sc.affected, affected, n);
    inc_refinement(E, L, cc_same_community != 0);
    down(E, s, L.s_cur.p, n);
    down(E, refined, E.sc.refined.p, n);
    E.sync();
  });
}

hl_status hl_dbg_set_exact_tfilter(int32_t on) {
  g_exact_tfilter.store(on ? 1 : 0);
  return HL_OK;
}

hl_status hl_dbg_set_bins(uint32_t mid_max, uint32_t wide_max) {
  if ((mid_max && (mid_max < 33 || mid_max > 128)) ||
      (wide_max && (wide_max > 512 || wide_max < (mid_max ? mid_max : 128)))) {
    g_err = "bins: mid_max in [33, 128], wide_max in [mid_max, 512] (0 = default)";
    return HL_ERR_INVALID_INPUT;
  }
  g_dbg_mid.store(mid_max);
  g_dbg_wide.store(wide_max);
  return HL_OK;
}

hl_status hl_dbg_set_bucket_slots(uint32_t slots) {
  g_pb_slots.store(slots);  // 0 (or out of range): the fold kernel's full table
  return HL_OK;
}

hl_status hl_dbg_set_hub_defer(uint32_t entries) {
  g_dbg_hub_defer.store(entries);  // 0: each handle's own (autotuned) bound
  return HL_OK;
}

hl_status hl_dbg_set_pb_round(uint64_t entries) {
  g_dbg_pb_round.store(entries);  // 0: the default round size
  return HL_OK;
}

hl_status hl_dbg_set_mode(uint32_t mode) {
  if (mode != HL_MODE_DETERMINISTIC && mode != HL_MODE_THROUGHPUT) {
    g_err = "mode must be HL_MODE_DETERMINISTIC or HL_MODE_THROUGHPUT";
    return HL_ERR_INVALID_INPUT;
  }
  g_dbg_mode.store(mode);
  return HL_OK;
}

hl_status hl_dbg_inc_aggregation(int32_t device, uint32_t n, const uint64_t* off,
                                 const uint32_t* col, const double* w, const uint32_t* dsrc,
                                 const uint32_t* ddst, const double* dw, uint64_t dk,
                                 const uint32_t* s_pre, const uint32_t* s_cur,
                                 const uint8_t* refined, int32_t changed_only,
                                 int32_t edge_weight_loops, uint32_t* out_s_pre,
                                 uint32_t* out_next_n, uint32_t* out_u, uint32_t* out_v,
                                 double* out_w, uint64_t cap, uint64_t* out_count) {
  HL_TRY({
    auto B = scratch_engine(device);
    Engine& E = *B->E;
    Level L;
    level_from_host(E, L, n, off, col, w);
    up(E, L.s_pre, s_pre, n);
    up(E, L.s_cur, s_cur, n);
    up(E, E.sc.refined, refined, n);
    DevEdges D = edges_up(E, B->bb, dsrc, ddst, dw, dk);
    u32 nn = 0;
    u64 cnt = inc_aggregation(E, L, D, &nn, changed_only != 0, edge_weight_loops != 0);
    *out_count = cnt;
    if (out_next_n) *out_next_n = nn;
    require(cnt <= cap, "output capacity too small");
    down(E, out_s_pre, L.s_pre.p, n);
    down(E, out_u, E.sc.eu2.p, cnt);
    down(E, out_v, E.sc.ev2.p, cnt);
    down(E, out_w, E.sc.ew2.p, cnt);
    E.sync();
  });
}

hl_status hl_dbg_modularity(int32_t device, uint32_t n, const uint64_t* off, const uint32_t* col,
                            const double* w, const uint32_t* part, double* q) {
  HL_TRY({
    auto B = scratch_engine(device);
    Engine& E = *B->E;
    Level L;
    level_from_host(E, L, n, off, col, w);
    DBuf<u32> pp;
    up(E, pp, part, n);
    *q = modularity(E, L, pp.p);
  });
}

hl_status hl_canonicalize(int32_t device, uint32_t* labels, uint64_t n) {
  HL_TRY({
    auto B = scratch_engine(device);
    Engine& E = *B->E;
    DBuf<u32> a, b;
    up(E, a, labels, n);
    b.ensure(E.mem, n ? n : 1);
    canonicalize_device(E, a.p, n, b.p);
    down(E, labels, b.p, n);
    E.sync();
  });
}

}  // extern "C"
