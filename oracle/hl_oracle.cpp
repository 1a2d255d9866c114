// hl_oracle.cpp — CPU ORACLE (test infrastructure only).
//
// A plain C++ restatement of the HIT-Leiden incremental update path of the
// Rust crate `hit_leiden` 0.1.0.  It exists so that the CUDA path can be
// checked against the reference's algorithm on the same inputs; it is never
// linked into, called by, or used as a fallback of the product library.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
//
// Parity anchors: every function cites the reference file:line it restates.
// The reference cannot be built here (Rust; no cargo/rustc), so the oracle is
// pinned against the reference's own unit-test known answers (restated in
// tests/test_oracle_kat.py) rather than against a live reference run.
//
// Canonical choices where the reference's result depends on ahash iteration
// order (randomised per process) or on thread_rng:
//   * CSR rows are kept sorted by ascending neighbour id (the reference keeps
//     insertion order in `From` and hash order after `apply_delta`).
//   * "First encountered in CSR order" replaces HashMap iteration order when
//     scanning neighbour communities / sub-communities (ties keep the earliest).
//   * Affected sub-communities are processed in ascending id order when new
//     sub-community ids are handed out (reference: hash order).
//   * Compressed ΔH (inc-aggregation) is emitted in ascending (u,v) order.
//   * 2m is the fixed pairwise tree sum of the per-vertex row sums (tile 1024,
//     stride-halving); the reference sums all CSR weights left to right.  For
//     integer weights every order gives the same bits.
//   * Community ids that reached >= n (empty-community ids n+v) are compacted
//     by rank at the start of inc-movement; the reference would index out of
//     bounds there (`community_degrees` sized n, hit_leiden.rs:1060-1066).
//   * run()'s thread_rng shuffle is replaced by a seeded splitmix64 shuffle.
//
// Build: oracle/Makefile (g++ -O3 -ffp-contract=off, so that a*b+c is never
// fused: the gain formulas must round exactly like the reference's f64 code).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <set>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include <atomic>
#include <thread>

extern "C" {
#include "hl_oracle.h"
}

namespace ora {

// ---------------------------------------------------------------------------
// Host threads for the throughput mode's snapshot evaluations (the reference
// runs them on rayon's pool).  Work is taken in chunks from a shared counter;
// each worker builds its own scratch.  Results are written by index, so they do
// not depend on the number of threads.
// ---------------------------------------------------------------------------
static std::atomic<int> g_threads{0};  // 0 = hardware concurrency, at most 64

static int num_threads() {
  int t = g_threads.load();
  if (t <= 0) {
    t = (int)std::thread::hardware_concurrency();
    if (t <= 0) t = 1;
    if (t > 64) t = 64;
  }
  return t;
}

template <typename MakeScratch, typename Body>
static void parallel_for(size_t count, MakeScratch make, Body body) {
  const int nt = (int)std::min<size_t>((size_t)num_threads(), (count + 255) / 256);
  if (nt <= 1) {
    auto sc = make();
    for (size_t i = 0; i < count; ++i) body(i, sc);
    return;
  }
  std::atomic<size_t> next{0};
  auto worker = [&]() {
    auto sc = make();
    for (;;) {
      const size_t a = next.fetch_add(256);
      if (a >= count) break;
      const size_t b = std::min(count, a + 256);
      for (size_t i = a; i < b; ++i) body(i, sc);
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
  worker();
  for (std::thread& th : pool) th.join();
}

using u32 = uint32_t;
using u64 = uint64_t;

// ---------------------------------------------------------------------------
// Graph: undirected weighted CSR, both directions stored, a self-loop stored
// twice in its own row (in_memory.rs:30-72).  Rows sorted by neighbour id.
// ---------------------------------------------------------------------------
struct Graph {
  u32 n = 0;
  std::vector<u64> off{0};
  std::vector<u32> col;
  std::vector<double> w;

  u64 deg(u32 v) const { return off[v + 1] - off[v]; }
};

struct Edge {
  u32 u, v;
  double w;
};

// in_memory.rs:30-72 (`From<&GraphInput>`), rows then sorted by neighbour id
// (stable, so duplicate input edges keep their input order).
static Graph graph_from_edges(u32 n, const std::vector<Edge>& edges) {
  Graph g;
  g.n = n;
  std::vector<u64> degree(n, 0);
  for (const Edge& e : edges) {
    degree[e.u] += 1;
    degree[e.v] += 1;
  }
  g.off.assign(n + 1, 0);
  for (u32 i = 0; i < n; ++i) g.off[i + 1] = g.off[i] + degree[i];
  g.col.assign(g.off[n], 0);
  g.w.assign(g.off[n], 0.0);
  std::vector<u64> cur(g.off.begin(), g.off.end() - 1);
  for (const Edge& e : edges) {
    u64 a = cur[e.u]++;
    g.col[a] = e.v;
    g.w[a] = e.w;
    u64 b = cur[e.v]++;
    g.col[b] = e.u;
    g.w[b] = e.w;
  }
  std::vector<std::pair<u32, double>> row;
  for (u32 i = 0; i < n; ++i) {
    row.clear();
    for (u64 p = g.off[i]; p < g.off[i + 1]; ++p) row.push_back({g.col[p], g.w[p]});
    std::stable_sort(row.begin(), row.end(),
                     [](const std::pair<u32, double>& a, const std::pair<u32, double>& b) {
                       return a.first < b.first;
                     });
    for (u64 p = g.off[i], j = 0; p < g.off[i + 1]; ++p, ++j) {
      g.col[p] = row[j].first;
      g.w[p] = row[j].second;
    }
  }
  return g;
}

// in_memory.rs:103-137 (`apply_delta`, `collect_canonical_edges`,
// `apply_delta_edges`).  `keep_self_loops=false` reproduces the reference:
// collect_canonical_edges keeps `node < neighbor` only (:125), so every
// existing self-loop is dropped; self-loops carried by the delta survive.
static Graph apply_delta(const Graph& g, u32 delta_n, const std::vector<Edge>& delta,
                         bool keep_self_loops) {
  // Existing canonical edges, already in ascending (u, v) order because rows
  // are sorted and scanned in node order; a repeated key keeps the last
  // weight, as HashMap::insert does.
  struct KW {
    u64 key;
    double w;
  };
  std::vector<KW> ex;
  ex.reserve(g.col.size() / 2 + 1);
  for (u32 v = 0; v < g.n; ++v) {
    for (u64 p = g.off[v]; p < g.off[v + 1]; ++p) {
      u32 nb = g.col[p];
      if (v < nb || (keep_self_loops && v == nb)) {
        u64 key = ((u64)v << 32) | nb;
        if (!ex.empty() && ex.back().key == key)
          ex.back().w = g.w[p];
        else
          ex.push_back({key, g.w[p]});
      }
    }
  }
  // Delta keys in batch order, stably sorted by key.
  std::vector<std::pair<u64, u64>> dk(delta.size());
  for (size_t i = 0; i < delta.size(); ++i) {
    u32 a = std::min(delta[i].u, delta[i].v), b = std::max(delta[i].u, delta[i].v);
    dk[i] = {((u64)a << 32) | b, (u64)i};
  }
  std::stable_sort(dk.begin(), dk.end(),
                   [](const std::pair<u64, u64>& x, const std::pair<u64, u64>& y) {
                     return x.first < y.first;
                   });
  std::vector<Edge> edges;
  edges.reserve(ex.size() + dk.size());
  size_t i = 0, j = 0;
  while (i < ex.size() || j < dk.size()) {
    u64 key;
    double x;
    if (j >= dk.size() || (i < ex.size() && ex[i].key < dk[j].first)) {
      key = ex[i].key;
      x = ex[i].w;
      ++i;
    } else {
      key = dk[j].first;
      x = 0.0;
      if (i < ex.size() && ex[i].key == key) {
        x = ex[i].w;
        ++i;
      }
      while (j < dk.size() && dk[j].first == key) {
        x += delta[dk[j].second].w;  // existing weight first, then batch order
        ++j;
      }
    }
    if (x > 1e-12) edges.push_back({(u32)(key >> 32), (u32)key, x});
  }
  u32 n = std::max(g.n, delta_n);
  return graph_from_edges(n, edges);
}

// Sum records per (min, max) key in push order; ascending key output.
static std::vector<Edge> compress_sum(const std::vector<Edge>& recs, double threshold) {
  std::vector<std::pair<u64, u64>> idx(recs.size());
  for (size_t i = 0; i < recs.size(); ++i) {
    u32 a = std::min(recs[i].u, recs[i].v), b = std::max(recs[i].u, recs[i].v);
    idx[i] = {((u64)a << 32) | b, (u64)i};
  }
  std::stable_sort(idx.begin(), idx.end(),
                   [](const std::pair<u64, u64>& x, const std::pair<u64, u64>& y) {
                     return x.first < y.first;
                   });
  std::vector<Edge> out;
  for (size_t t = 0; t < idx.size();) {
    u64 key = idx[t].first;
    double x = 0.0;
    while (t < idx.size() && idx[t].first == key) x += recs[idx[t++].second].w;
    if (std::fabs(x) > threshold) out.push_back({(u32)(key >> 32), (u32)key, x});
  }
  return out;
}

// Per-vertex weighted degree: left-to-right sum over the row in CSR order
// (hit_leiden.rs:1063 `graph.neighbors(i).map(|(_, w)| w).sum()`).
static std::vector<double> node_degrees(const Graph& g) {
  std::vector<double> k(g.n, 0.0);
  for (u32 v = 0; v < g.n; ++v) {
    double s = 0.0;
    for (u64 p = g.off[v]; p < g.off[v + 1]; ++p) s += g.w[p];
    k[v] = s;
  }
  return k;
}

// Fixed-shape pairwise sum (the canonical 2m): tiles of 1024 values padded
// with +0.0, each tile folded by stride halving (x[i] += x[i+s], s = 512..1),
// then the tile sums are folded the same way until one value remains.
static double tree_sum(std::vector<double> x) {
  const size_t T = 1024;
  if (x.empty()) return 0.0;
  while (true) {
    size_t tiles = (x.size() + T - 1) / T;
    std::vector<double> part(tiles, 0.0);
    double buf[T];
    for (size_t t = 0; t < tiles; ++t) {
      for (size_t i = 0; i < T; ++i) {
        size_t idx = t * T + i;
        buf[i] = idx < x.size() ? x[idx] : 0.0;
      }
      for (size_t s = T / 2; s >= 1; s >>= 1)
        for (size_t i = 0; i < s; ++i) buf[i] = buf[i] + buf[i + s];
      part[t] = buf[0];
    }
    if (tiles == 1) return part[0];
    x.swap(part);
  }
}

static double twice_total_weight(const std::vector<double>& k) { return tree_sum(k); }

// hit_leiden.rs:121-161 (`compute_modularity`) on an edge list: the form the
// reference's own tests call.
static double modularity_edges(u32 n, const std::vector<Edge>& edges, const u32* part) {
  std::vector<double> kd(n, 0.0);
  double total = 0.0;
  for (const Edge& e : edges) {
    kd[e.u] += e.w;
    kd[e.v] += e.w;
    total += e.w;
  }
  double twice_m = total * 2.0;
  if (twice_m == 0.0) return 0.0;
  double intra = 0.0;
  for (const Edge& e : edges)
    if (part[e.u] == part[e.v]) intra += e.w * 2.0;
  std::map<u32, double> cds;
  for (u32 i = 0; i < n; ++i) cds[part[i]] += kd[i];
  double expected = 0.0;
  for (const auto& kv : cds) expected += kv.second * kv.second / twice_m;
  return (intra - expected) / twice_m;
}

// Same quantity on the resident CSR (each edge appears twice there, a
// self-loop twice in its row): intra and degrees agree with the edge-list form.
// The per-community totals are the reference's node-order sums; the two outer
// sums are accumulated in long double (the reference adds them in hash order,
// so only their accurately rounded value is order-free).
static double modularity_csr(const Graph& g, const u32* part) {
  std::vector<double> k = node_degrees(g);
  double tw = twice_total_weight(k);
  if (tw == 0.0) return 0.0;
  long double intra = 0.0L;
  for (u32 v = 0; v < g.n; ++v)
    for (u64 p = g.off[v]; p < g.off[v + 1]; ++p)
      if (part[v] == part[g.col[p]]) intra += g.w[p];
  u32 mx = 0;
  for (u32 i = 0; i < g.n; ++i) mx = std::max(mx, part[i]);
  std::vector<double> cds((size_t)mx + 1, 0.0);
  std::vector<uint8_t> seen((size_t)mx + 1, 0);
  for (u32 i = 0; i < g.n; ++i) {
    cds[part[i]] += k[i];
    seen[part[i]] = 1;
  }
  long double expected = 0.0L;
  for (size_t c = 0; c < cds.size(); ++c)
    if (seen[c]) expected += (long double)(cds[c] * cds[c] / tw);
  return (double)((intra - expected) / (long double)tw);
}

// hit_leiden.rs:358-376: first-seen contiguous relabel.
static void canonicalize(std::vector<u32>& c) {
  std::unordered_map<u32, u32> remap;
  u32 next = 0;
  for (u32& x : c) {
    auto it = remap.find(x);
    if (it == remap.end()) it = remap.emplace(x, next++).first;
    x = it->second;
  }
}

static size_t count_unique(const std::vector<u32>& v) {
  std::unordered_set<u32> s(v.begin(), v.end());
  return s.size();
}

// ΔQ(v: C -> C', γ) exactly as written in the reference
// (parallel_frontier.rs:185-190, hit_leiden.rs:1135-1140).
static inline double move_gain(double w_to, double w_cur, double tw, double gamma, double kv,
                               double d_cur, double d_to) {
  return (w_to - w_cur) / tw + gamma * kv * (d_cur - kv - d_to) / (tw * tw);
}
// Gain of moving to the empty community (parallel_frontier.rs:207-211).
static inline double empty_gain(double w_cur, double tw, double gamma, double kv, double d_cur) {
  return -w_cur / tw + gamma * kv * (d_cur - kv) / (tw * tw);
}

struct Move {
  u32 node, from, to;
  double kdeg, gain;
};

// throughput.rs:204-236 (`select_decoupled_moves`): sort by gain desc then
// node asc; greedily accept iff from ∉ acceptors and to ∉ emitters.
static std::vector<Move> select_decoupled(std::vector<Move> c) {
  std::stable_sort(c.begin(), c.end(), [](const Move& a, const Move& b) {
    if (a.gain > b.gain) return true;
    if (a.gain < b.gain) return false;
    return a.node < b.node;
  });
  std::unordered_set<u32> emit, acc, moved;
  std::vector<Move> sel;
  for (const Move& m : c) {
    if (m.gain <= 0.0) continue;
    if (moved.count(m.node)) continue;
    if (acc.count(m.from) || emit.count(m.to)) continue;
    sel.push_back(m);
    moved.insert(m.node);
    emit.insert(m.from);
    acc.insert(m.to);
  }
  return sel;
}

// Per-vertex best move on a fixed snapshot: parallel_frontier.rs:150-235
// (`execute_shard` body for one node).  Returns gain 0 / to = from when no
// positive move exists.
struct Eval {
  u32 to;
  double gain;
};

struct MoveScratch {
  std::vector<double> buf;
  std::vector<u32> dirty;
};

static Eval eval_move(const Graph& g, u32 v, const std::vector<u32>& f, const std::vector<double>& d,
                      const std::vector<double>& k, double tw, double gamma, bool allow_empty,
                      MoveScratch& sc) {
  u32 cur = f[v];
  double kv = k[v];
  u32 best = cur;
  double bestg = 0.0;
  double wcur = 0.0;
  for (u64 p = g.off[v]; p < g.off[v + 1]; ++p) {
    u32 nb = g.col[p];
    if (nb == v) continue;
    u32 c = f[nb];
    if (sc.buf[c] == 0.0) sc.dirty.push_back(c);
    sc.buf[c] += g.w[p];
    if (c == cur) wcur += g.w[p];
  }
  double dcur = d[cur];
  for (u32 c : sc.dirty) {
    if (c == cur) continue;
    double gn = move_gain(sc.buf[c], wcur, tw, gamma, kv, dcur, d[c]);
    if (gn > bestg) {
      bestg = gn;
      best = c;
    }
  }
  if (allow_empty) {
    double eg = empty_gain(wcur, tw, gamma, kv, dcur);
    if (eg > bestg) {
      bestg = eg;
      best = g.n + v;
    }
  }
  for (u32 c : sc.dirty) sc.buf[c] = 0.0;
  sc.dirty.clear();
  return {best, bestg};
}

// Rank-compaction of community ids when any id reached >= n.
static void compact_ids_if_needed(std::vector<u32>& f, u32 n) {
  u32 mx = 0;
  for (u32 x : f) mx = std::max(mx, x);
  if (f.empty() || mx < n) return;
  std::vector<u32> ids(f.begin(), f.end());
  std::sort(ids.begin(), ids.end());
  ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
  for (u32& x : f) x = (u32)(std::lower_bound(ids.begin(), ids.end(), x) - ids.begin());
}

struct MoveOut {
  std::vector<uint8_t> changed, affected;
  u32 iterations = 0;
  u64 rounds_candidates = 0, rounds_moves = 0, traversed = 0;
};

// hit_leiden.rs:1024-1192 (`inc_movement`) with the throughput branch
// (:1068-1101 → throughput.rs:80-202) and the deterministic branch
// (:1103-1191).
// ---------------------------------------------------------------------------
// Round-to-round hub key sums (OR_FLAG_HUB_CHECK; test infrastructure, not a
// restatement of the reference).  Between two throughput rounds only the
// moved vertices' labels change, so a long row's per-key weight sums can be
// kept and corrected by its moved neighbours instead of being recomputed.
// The table keeps, per key, the sum, the first CSR position, and whether that
// position may be out of date (its entry moved to another key); it is
// recomputed only when the key ties the best gain, the one place the tie
// rule reads it.  Exact for integral weights, where sums do not depend on the
// order of additions; the check compares every such evaluation with the full
// one (eval_move).
// ---------------------------------------------------------------------------
constexpr u64 HUB_CHECK_DEG = 512;
static std::atomic<unsigned long long> g_hub_check[6];  // see or_hub_check_counters

struct HubCheck {
  struct Ent {
    double sum;
    u64 first;
    bool stale;
  };
  const Graph& g;
  std::unordered_map<u32, std::unordered_map<u32, Ent>> tabs;
  explicit HubCheck(const Graph& gr) : g(gr) {}

  u64 first_pos(u32 v, u32 key, const std::vector<u32>& f) const {
    for (u64 q = g.off[v]; q < g.off[v + 1]; ++q)
      if (g.col[q] != v && f[g.col[q]] == key) return q - g.off[v];
    return ~0ull;
  }

  // The evaluation eval_move makes (empty community allowed), from v's table.
  Eval eval(u32 v, const std::vector<u32>& f, const std::vector<double>& d,
            const std::vector<double>& k, double tw, double gamma) {
    auto it = tabs.find(v);
    if (it == tabs.end()) {
      std::unordered_map<u32, Ent> tb;
      for (u64 q = g.off[v]; q < g.off[v + 1]; ++q) {
        const u32 nb = g.col[q];
        if (nb == v) continue;
        auto r = tb.find(f[nb]);
        if (r == tb.end()) tb[f[nb]] = Ent{g.w[q], q - g.off[v], false};
        else r->second.sum += g.w[q];
      }
      it = tabs.emplace(v, std::move(tb)).first;
      ++g_hub_check[4];
    }
    auto& tb = it->second;
    const u32 cur = f[v];
    const double kv = k[v];
    auto rc = tb.find(cur);
    const double wcur = rc == tb.end() ? 0.0 : rc->second.sum;
    const double dcur = d[cur];
    u32 best = cur;
    double bestg = 0.0;
    for (auto& kvp : tb) {
      ++g_hub_check[5];
      const u32 c = kvp.first;
      Ent& e = kvp.second;
      if (c == cur || e.sum == 0.0) continue;
      const double gn = move_gain(e.sum, wcur, tw, gamma, kv, dcur, d[c]);
      if (gn <= bestg && !(gn == bestg && gn > 0.0)) continue;
      if (gn == bestg) {  // a tie: the first position decides
        for (Ent* x : {&e, &tb[best]})
          if (x->stale) {
            x->first = first_pos(v, x == &e ? c : best, f);
            x->stale = false;
            ++g_hub_check[2];
          }
        if (e.first < tb[best].first) best = c;
        continue;
      }
      bestg = gn;
      best = c;
    }
    const double eg = empty_gain(wcur, tw, gamma, kv, dcur);
    if (eg > bestg) {
      bestg = eg;
      best = g.n + v;
    }
    return {best, bestg};
  }

  // The round's accepted moves: each moved vertex's entry in the tables of
  // its neighbours, found by binary search (rows are sorted by neighbour).
  void correct(const std::vector<Move>& sel) {
    for (const Move& m : sel) {
      for (u64 pm = g.off[m.node]; pm < g.off[m.node + 1]; ++pm) {
        const u32 h = g.col[pm];
        if (h == m.node) continue;
        auto ih = tabs.find(h);
        if (ih == tabs.end()) continue;
        u64 lo = g.off[h], hi = g.off[h + 1];
        while (hi - lo > 1) {
          const u64 mid = (lo + hi) / 2;
          if (g.col[mid] <= m.node) lo = mid;
          else hi = mid;
        }
        const u64 q = lo - g.off[h];
        const double w = g.w[lo];
        auto& tb = ih->second;
        Ent& ef = tb[m.from];
        ef.sum -= w;
        if (!ef.stale && ef.first == q) ef.stale = true;
        auto rt = tb.find(m.to);
        if (rt == tb.end() || rt->second.sum == 0.0) {
          tb[m.to] = Ent{w, q, false};
        } else {
          rt->second.sum += w;
          if (!rt->second.stale) rt->second.first = std::min(rt->second.first, q);
        }
        ++g_hub_check[3];
      }
    }
  }
};

// A fixed case for the stale first position: hub 0 with unit edges to 1..7;
// communities 10 = {1, 2, 7} and 20 = {3, 4} of equal degree.  Vertex 1 (the
// first entry of key 10) moves to 40, so 10's first position goes stale and
// 10 and 20 then tie (two entries each): the tie rule needs 10's true first
// position (vertex 2) to pick 10.  Returns the rescans made, or -1 when an
// evaluation differs from eval_move.
static int hub_check_selftest() {
  std::vector<Edge> e;
  for (u32 x = 1; x <= 7; ++x) e.push_back({0, x, 1.0});
  const Graph g = graph_from_edges(50, e);
  std::vector<u32> f(50);
  for (u32 x = 0; x < 50; ++x) f[x] = x;
  f[1] = f[2] = f[7] = 10;
  f[3] = f[4] = 20;
  const std::vector<double> k = node_degrees(g);
  const double tw = twice_total_weight(k);
  std::vector<double> d(101, 0.0);
  d[10] = d[20] = 3.0;
  d[0] = k[0];
  d[5] = d[6] = 10.0;  // the singletons 5 and 6 and the new community 40 lose
  d[40] = 5.0;
  MoveScratch sc;
  sc.buf.assign(d.size() + g.n + 1, 0.0);
  HubCheck hub(g);
  const unsigned long long r0 = g_hub_check[2].load();
  Eval a = hub.eval(0, f, d, k, tw, 1.0);
  Eval b = eval_move(g, 0, f, d, k, tw, 1.0, true, sc);
  if (a.to != b.to || a.gain != b.gain) return -1;
  f[1] = 40;
  hub.correct({Move{1, 10, 40, k[1], 0.0}});
  a = hub.eval(0, f, d, k, tw, 1.0);
  b = eval_move(g, 0, f, d, k, tw, 1.0, true, sc);
  if (a.to != b.to || a.gain != b.gain || a.to != 10) return -1;
  return (int)(g_hub_check[2].load() - r0);
}

static MoveOut inc_movement(const Graph& g, const std::vector<Edge>& delta, std::vector<u32>& f,
                            const std::vector<u32>& s, double gamma, int mode, u32 max_rounds,
                            bool compact, bool mark_moved = false,
                            const std::vector<u32>* extra_k = nullptr, u64 hub_check_deg = 0) {
  u32 n = g.n;
  MoveOut out;
  out.changed.assign(n, 0);
  out.affected.assign(n, 0);
  std::vector<uint8_t> active(n, 0);
  for (const Edge& e : delta) {
    double a = e.w;
    if (a > 0.0 && f[e.u] != f[e.v]) active[e.u] = active[e.v] = 1;
    if (a < 0.0 && f[e.u] == f[e.v]) active[e.u] = active[e.v] = 1;
    if (s[e.u] == s[e.v]) out.affected[e.u] = out.affected[e.v] = 1;
  }
  if (delta.empty()) std::fill(active.begin(), active.end(), 1);
  // M8 (multi-level): the nodes this level gained from splits at the level
  // below join K, so the sub-community they inherited (M6) is split again
  // when they are not connected to it.
  if (extra_k)
    for (u32 x : *extra_k)
      if (x < n) out.affected[x] = 1;
  if (compact) compact_ids_if_needed(f, n);

  std::vector<double> k = node_degrees(g);
  double tw = twice_total_weight(k);
  std::vector<double> d(2 * (size_t)n + 1, 0.0);
  for (u32 i = 0; i < n; ++i) {
    if (f[i] >= d.size()) d.resize((size_t)f[i] + 1, 0.0);
    d[f[i]] += k[i];
  }

  if (mode == OR_MODE_THROUGHPUT) {
    std::vector<u32> act;
    for (u32 i = 0; i < n; ++i)
      if (active[i]) act.push_back(i);
    u32 it = 0;
    std::vector<Eval> ev;
    std::unique_ptr<HubCheck> hub;
    if (hub_check_deg) hub.reset(new HubCheck(g));
    while (!act.empty() && it < max_rounds) {
      // Every active vertex is evaluated on the same snapshot (the reference
      // runs these with rayon, throughput.rs:80-202), so the evaluations run
      // in parallel; candidates are then taken in list order.
      ev.assign(act.size(), Eval{0, 0.0});
      const size_t bufsize = d.size() + n + 1;
      parallel_for(
          act.size(),
          [&]() {
            MoveScratch tsc;
            tsc.buf.assign(bufsize, 0.0);
            return tsc;
          },
          [&](size_t i, MoveScratch& tsc) {
            ev[i] = eval_move(g, act[i], f, d, k, tw, gamma, true, tsc);
          });
      if (hub) {
        for (size_t i = 0; i < act.size(); ++i) {
          if (g.deg(act[i]) <= hub_check_deg) continue;
          const Eval e = hub->eval(act[i], f, d, k, tw, gamma);
          ++g_hub_check[0];
          if (e.to != ev[i].to || e.gain != ev[i].gain) ++g_hub_check[1];
        }
      }
      std::vector<Move> cand;
      for (size_t i = 0; i < act.size(); ++i) {
        const u32 v = act[i];
        out.traversed += g.deg(v);
        if (ev[i].gain <= 0.0) continue;
        cand.push_back({v, f[v], ev[i].to, k[v], ev[i].gain});
      }
      out.rounds_candidates += cand.size();
      std::vector<Move> sel = select_decoupled(cand);
      size_t need = 0;
      for (const Move& m : sel) need = std::max(need, (size_t)m.to + 1);
      if (need > d.size()) d.resize(need, 0.0);
      double total = 0.0;
      for (const Move& m : sel) total += m.gain;
      std::vector<uint8_t> next(n, 0);
      act.clear();
      if (total <= 0.0) {
        ++it;
        break;
      }
      for (const Move& m : sel) {
        f[m.node] = m.to;
        d[m.from] -= m.kdeg;
        d[m.to] += m.kdeg;
        out.changed[m.node] = 1;
        if (mark_moved) out.affected[m.node] = 1;
      }
      out.rounds_moves += sel.size();
      if (hub) hub->correct(sel);
      for (const Move& m : sel) {
        for (u64 p = g.off[m.node]; p < g.off[m.node + 1]; ++p) {
          u32 nb = g.col[p];
          if (f[nb] != m.to) next[nb] = 1;
          if (s[m.node] == s[nb]) out.affected[m.node] = out.affected[nb] = 1;
        }
      }
      for (u32 i = 0; i < n; ++i)
        if (next[i]) act.push_back(i);
      ++it;
    }
    out.iterations = it;
    return out;
  }

  // Deterministic (sequential Gauss–Seidel): pop the lowest active index
  // (:1109), accumulate Σw per neighbour community *including* self-loops
  // (:1119-1125), strict '>' in first-encounter order, then the empty
  // community with id `next_empty` (:1104, :1150-1162).  The reference starts
  // it at the length of its community-degree array, n (:1060); `d` here is
  // longer, to hold the throughput path's ids n + v.  An existing id >= n
  // (a state the reference cannot reach, where it would index out of bounds)
  // moves the start past it.
  std::set<u32> aset;
  for (u32 i = 0; i < n; ++i)
    if (active[i]) aset.insert(i);
  size_t next_empty = n;
  for (u32 x : f)
    if ((size_t)x >= next_empty) next_empty = (size_t)x + 1;
  std::vector<double> buf(d.size() + 1, 0.0);
  std::vector<u32> order;
  std::vector<uint8_t> seen(d.size() + 1, 0);
  while (!aset.empty()) {
    u32 v = *aset.begin();
    aset.erase(aset.begin());
    out.traversed += g.deg(v);
    u32 cur = f[v];
    u32 best = cur;
    double bestg = 0.0;
    double wcur = 0.0;
    double kv = k[v];
    order.clear();
    for (u64 p = g.off[v]; p < g.off[v + 1]; ++p) {
      u32 c = f[g.col[p]];
      if (c >= buf.size()) {
        buf.resize((size_t)c + 1, 0.0);
        seen.resize((size_t)c + 1, 0);
      }
      if (!seen[c]) {
        seen[c] = 1;
        order.push_back(c);
      }
      buf[c] += g.w[p];
      if (c == cur) wcur += g.w[p];
    }
    for (u32 c : order) {
      if (c == cur) continue;
      double gn = move_gain(buf[c], wcur, tw, gamma, kv, d[cur], d[c]);
      if (gn > bestg) {
        bestg = gn;
        best = c;
      }
    }
    {
      double eg = empty_gain(wcur, tw, gamma, kv, d[cur]);
      if (eg > bestg) {
        bestg = eg;
        best = (u32)next_empty;
      }
    }
    for (u32 c : order) {
      buf[c] = 0.0;
      seen[c] = 0;
    }
    if (bestg <= 0.0) continue;
    u32 old = f[v];
    // An empty-community move allocates next_empty and moves the counter on
    // (:1170-1173: the reference's array grows by one, and its length is the
    // next id).
    if ((size_t)best == next_empty) next_empty = (size_t)best + 1;
    if (best >= d.size()) {
      d.resize((size_t)best + 1, 0.0);
      if (buf.size() < d.size()) {
        buf.resize(d.size(), 0.0);
        seen.resize(d.size(), 0);
      }
    }
    f[v] = best;
    out.changed[v] = 1;
    if (mark_moved) out.affected[v] = 1;
    d[old] -= kv;
    d[best] += kv;
    ++out.rounds_moves;
    for (u64 p = g.off[v]; p < g.off[v + 1]; ++p) {
      u32 nb = g.col[p];
      if (f[nb] != best) aset.insert(nb);
      if (s[v] == s[nb]) out.affected[v] = out.affected[nb] = 1;
    }
  }
  out.iterations = 1;
  return out;
}

// Connected components of one sub-community over edges whose both ends carry
// that sub-community id (hit_leiden.rs:1194-1243): BFS from each unvisited
// member in ascending order, so components come out ordered by their minimum.
static std::vector<std::vector<u32>> cc_by_subcommunity(const Graph& g,
                                                        const std::vector<u32>& verts,
                                                        const std::vector<u32>& s,
                                                        std::vector<uint8_t>& visited,
                                                        const std::vector<u32>* f = nullptr) {
  std::vector<std::vector<u32>> comps;
  std::deque<u32> q;
  for (u32 st : verts) {
    if (visited[st]) continue;
    std::vector<u32> comp;
    q.push_back(st);
    visited[st] = 1;
    while (!q.empty()) {
      u32 c = q.front();
      q.pop_front();
      comp.push_back(c);
      u32 sc = s[c];
      for (u64 p = g.off[c]; p < g.off[c + 1]; ++p) {
        u32 nb = g.col[p];
        if (s[nb] == sc && !visited[nb] && (!f || (*f)[nb] == (*f)[c])) {
          visited[nb] = 1;
          q.push_back(nb);
        }
      }
    }
    comps.push_back(std::move(comp));
  }
  return comps;
}

struct RefineOut {
  std::vector<uint8_t> refined;
  std::vector<std::pair<u32, u32>> new_ids;  // (new sub-community id, id it split from)
  u64 splits = 0, merges = 0;
};

// hit_leiden.rs:1554-1637 (`compute_blocked_subcommunities`): a candidate S is
// blocked when ΔQ(S→∅) = -w(S,C)/2m + γ d_S (d_C - d_S)/(2m)^2 > 1e-9.
// `faithful` keeps the reference's O(n) scans per candidate (timing only).
static std::vector<uint8_t> compute_blocked(const Graph& g, const std::vector<u32>& f,
                                            const std::vector<u32>& s,
                                            const std::vector<double>& dS,
                                            const std::vector<u32>& r_sorted,
                                            const std::vector<u64>& sizes,
                                            const std::vector<double>& k, double tw,
                                            double gamma, bool faithful) {
  u32 n = g.n;
  std::vector<uint8_t> cand(dS.size(), 0);
  std::vector<u32> cand_list;
  for (u32 v : r_sorted) {
    if (s[v] >= sizes.size() || sizes[s[v]] != 1) continue;
    u32 pc = f[v];
    for (u64 p = g.off[v]; p < g.off[v + 1]; ++p) {
      u32 nb = g.col[p];
      if (f[nb] != pc) continue;
      u32 ns = s[nb];
      if (ns != s[v] && !cand[ns]) {
        cand[ns] = 1;
        cand_list.push_back(ns);
      }
    }
  }
  std::vector<uint8_t> blocked(dS.size(), 0);
  if (cand_list.empty()) return blocked;
  u32 fmax = 0;
  for (u32 i = 0; i < n; ++i) fmax = std::max(fmax, f[i]);
  std::vector<double> dcomm((size_t)fmax + 1, 0.0);
  for (u32 i = 0; i < n; ++i) dcomm[f[i]] += k[i];
  // Members of every candidate, ascending.
  std::vector<u32> mstart(dS.size() + 1, 0), mlist;
  if (!faithful) {
    for (u32 i = 0; i < n; ++i)
      if (cand[s[i]]) mstart[s[i] + 1] += 1;
    for (size_t c = 0; c < dS.size(); ++c) mstart[c + 1] += mstart[c];
    mlist.assign(mstart.back(), 0);
    std::vector<u32> fill(mstart.begin(), mstart.end() - 1);
    for (u32 i = 0; i < n; ++i)
      if (cand[s[i]]) mlist[fill[s[i]]++] = i;
  }
  std::sort(cand_list.begin(), cand_list.end());
  for (u32 S : cand_list) {
    double ds = dS[S];
    if (ds <= 0.0) continue;
    std::vector<u32> mem;
    if (faithful) {
      for (u32 i = 0; i < n; ++i)
        if (s[i] == S) mem.push_back(i);
    } else {
      mem.assign(mlist.begin() + mstart[S], mlist.begin() + mstart[S + 1]);
    }
    u32 parent = mem.empty() ? 0 : f[mem[0]];
    double dpar = parent < dcomm.size() ? dcomm[parent] : 0.0;
    double wsp = 0.0;
    for (u32 i : mem)
      for (u64 p = g.off[i]; p < g.off[i + 1]; ++p)
        if (f[g.col[p]] == parent) wsp += g.w[p];
    double dq = -wsp / tw + gamma * ds * (dpar - ds) / (tw * tw);
    if (dq > 1e-9) blocked[S] = 1;
  }
  return blocked;
}

// throughput.rs:291-359 (`try_refinement_move`): same-community neighbours
// (self-loops included), first-encounter order, strict '>'.
struct RefMove {
  u32 node, from, to;
  double kdeg;
};

static bool try_refinement_move(const Graph& g, u32 v, const std::vector<u32>& f,
                                const std::vector<u32>& s, const std::vector<double>& dS,
                                const std::vector<double>& k, double tw, double gamma,
                                const std::vector<uint8_t>& blocked, std::vector<double>& buf,
                                std::vector<uint8_t>& seen, std::vector<u32>& order, RefMove& out) {
  u32 cc = f[v], cs = s[v];
  double kv = k[v];
  double wcur = 0.0;
  order.clear();
  for (u64 p = g.off[v]; p < g.off[v + 1]; ++p) {
    u32 nb = g.col[p];
    if (f[nb] != cc) continue;
    u32 sc = s[nb];
    if (!seen[sc]) {
      seen[sc] = 1;
      order.push_back(sc);
    }
    buf[sc] += g.w[p];
    if (sc == cs) wcur += g.w[p];
  }
  u32 best = cs;
  double bestg = 0.0;
  for (u32 c : order) {
    if (c == cs) continue;
    if (blocked[c]) continue;
    double gn = move_gain(buf[c], wcur, tw, gamma, kv, dS[cs], dS[c]);
    if (gn > bestg) {
      bestg = gn;
      best = c;
    }
  }
  for (u32 c : order) {
    buf[c] = 0.0;
    seen[c] = 0;
  }
  if (bestg > 0.0) {
    out = {v, cs, best, kv};
    return true;
  }
  return false;
}

// hit_leiden.rs:1514-1548 (`should_skip_candidate_t_filter`), O(n) scan.
static bool t_filter_skip(const Graph& g, u32 cand, u32 parent, const std::vector<u32>& s,
                          const std::vector<u32>& f, const std::vector<double>& dS, double dpar,
                          double tw, double gamma) {
  double ds = cand < dS.size() ? dS[cand] : 0.0;
  if (ds <= 0.0) return false;
  double wsp = 0.0;
  for (u32 i = 0; i < g.n; ++i) {
    if (s[i] != cand) continue;
    for (u64 p = g.off[i]; p < g.off[i + 1]; ++p)
      if (f[g.col[p]] == parent) wsp += g.w[p];
  }
  double dq = -wsp / tw + gamma * ds * (dpar - ds) / (tw * tw);
  return dq > 1e-9;
}

// hit_leiden.rs:1265-1416 (`inc_refinement`).
static RefineOut inc_refinement(const Graph& g, const std::vector<u32>& f, std::vector<u32>& s,
                                const std::vector<uint8_t>& affected, double gamma, int mode,
                                bool faithful, bool cc_same_community = false) {
  u32 n = g.n;
  RefineOut out;
  out.refined.assign(n, 0);
  // Affected sub-communities and their members (ascending).
  u32 mx = 0;
  for (u32 x : s) mx = std::max(mx, x);
  std::vector<uint8_t> aff((size_t)mx + 1, 0);
  for (u32 v = 0; v < n; ++v)
    if (affected[v]) aff[s[v]] = 1;
  // Members of each affected sub-community, ascending, grouped by id.
  std::vector<std::pair<u32, u32>> mem;
  for (u32 i = 0; i < n; ++i)
    if (aff[s[i]]) mem.push_back({s[i], i});
  std::stable_sort(mem.begin(), mem.end(),
                   [](const std::pair<u32, u32>& a, const std::pair<u32, u32>& b) {
                     return a.first < b.first;
                   });
  std::vector<std::pair<u32, std::vector<u32>>> nodes;
  for (size_t t = 0; t < mem.size();) {
    u32 S = mem[t].first;
    std::vector<u32> vs;
    while (t < mem.size() && mem[t].first == S) vs.push_back(mem[t++].second);
    nodes.push_back({S, std::move(vs)});
  }
  u64 next_id = n ? (u64)mx + 1 : 1;
  std::vector<uint8_t> visited(n, 0);
  for (auto& kv : nodes) {
    const std::vector<u32>& verts = kv.second;
    if (verts.empty()) continue;
    auto comps = cc_by_subcommunity(g, verts, s, visited, cc_same_community ? &f : nullptr);
    for (u32 v : verts) visited[v] = 0;
    if (comps.size() <= 1) continue;
    // Rust `max_by_key` keeps the last maximum.
    size_t largest = 0;
    for (size_t i = 0; i < comps.size(); ++i)
      if (comps[i].size() >= comps[largest].size()) largest = i;
    for (size_t i = 0; i < comps.size(); ++i) {
      if (i == largest) continue;
      u32 nid = (u32)next_id++;
      out.new_ids.push_back({nid, kv.first});
      for (u32 v : comps[i]) {
        s[v] = nid;
        out.refined[v] = 1;
      }
      ++out.splits;
    }
  }
  bool is_initial = true;
  for (u32 i = 0; i < n; ++i)
    if (s[i] != i) {
      is_initial = false;
      break;
    }
  if (is_initial) std::fill(out.refined.begin(), out.refined.end(), 1);

  u32 smax = 0;
  for (u32 x : s) smax = std::max(smax, x);
  std::vector<u64> sizes((size_t)smax + 1, 0);
  for (u32 x : s) sizes[x] += 1;
  std::vector<double> k = node_degrees(g);
  double tw = twice_total_weight(k);
  std::vector<double> dS((size_t)smax + 1, 0.0);
  for (u32 i = 0; i < n; ++i) dS[s[i]] += k[i];

  std::vector<u32> rs;
  for (u32 i = 0; i < n; ++i)
    if (out.refined[i]) rs.push_back(i);
  std::stable_sort(rs.begin(), rs.end(), [&](u32 a, u32 b) { return k[a] < k[b]; });

  std::vector<double> buf(dS.size(), 0.0);
  std::vector<uint8_t> seen(dS.size(), 0);
  std::vector<u32> order;

  if (mode == OR_MODE_THROUGHPUT) {
    std::vector<uint8_t> blocked = compute_blocked(g, f, s, dS, rs, sizes, k, tw, gamma, faithful);
    // Jacobi on the snapshot (throughput.rs:239-288): evaluated in parallel,
    // applied in list order.
    std::vector<RefMove> mv(rs.size());
    std::vector<uint8_t> has(rs.size(), 0);
    struct RefScratch {
      std::vector<double> buf;
      std::vector<uint8_t> seen;
      std::vector<u32> order;
    };
    parallel_for(
        rs.size(),
        [&]() {
          RefScratch t;
          t.buf.assign(dS.size(), 0.0);
          t.seen.assign(dS.size(), 0);
          return t;
        },
        [&](size_t i, RefScratch& t) {
          const u32 v = rs[i];
          if (sizes[s[v]] != 1) return;
          if (try_refinement_move(g, v, f, s, dS, k, tw, gamma, blocked, t.buf, t.seen, t.order,
                                  mv[i]))
            has[i] = 1;
        });
    std::vector<RefMove> upd;
    for (size_t i = 0; i < rs.size(); ++i)
      if (has[i]) upd.push_back(mv[i]);
    for (const RefMove& m : upd) {
      s[m.node] = m.to;
      dS[m.from] -= m.kdeg;
      dS[m.to] += m.kdeg;
      sizes[m.from] = sizes[m.from] ? sizes[m.from] - 1 : 0;
      sizes[m.to] += 1;
    }
    out.merges = upd.size();
    return out;
  }

  // Deterministic: hit_leiden.rs:1392-1413 → try_merge_singleton_refinement
  // (:1419-1511) with the live T-filter (:1514-1548).
  for (u32 v : rs) {
    if (sizes[s[v]] != 1) continue;
    u32 cc = f[v], cs = s[v];
    double kv = k[v];
    double wcur = 0.0;
    order.clear();
    for (u64 p = g.off[v]; p < g.off[v + 1]; ++p) {
      u32 nb = g.col[p];
      if (f[nb] != cc) continue;
      u32 sc = s[nb];
      if (!seen[sc]) {
        seen[sc] = 1;
        order.push_back(sc);
      }
      buf[sc] += g.w[p];
      if (sc == cs) wcur += g.w[p];
    }
    double dpar = 0.0;
    for (u32 i = 0; i < n; ++i)
      if (f[i] == cc) dpar += k[i];
    u32 best = cs;
    double bestg = 0.0;
    for (u32 c : order) {
      if (c == cs) continue;
      if (t_filter_skip(g, c, cc, s, f, dS, dpar, tw, gamma)) continue;
      double gn = move_gain(buf[c], wcur, tw, gamma, kv, dS[cs], dS[c]);
      if (gn > bestg) {
        bestg = gn;
        best = c;
      }
    }
    for (u32 c : order) {
      buf[c] = 0.0;
      seen[c] = 0;
    }
    if (bestg > 0.0) {
      s[v] = best;
      sizes[cs] -= 1;
      sizes[best] += 1;
      dS[cs] -= kv;
      dS[best] += kv;
      ++out.merges;
    }
  }
  return out;
}

// hit_leiden.rs:1639-1731 (`inc_aggregation`).  Options used only by the
// multi-level extension (the reference itself never aggregates: levels = 1):
//   changed_only      iterate R ∩ {s_cur != s_pre} (R holding unchanged nodes
//                      makes the reference emit a mixed pair twice)
//   edge_weight_loops  move the self-loop's edge weight w (the reference sums
//                      both CSR copies and moves 2w, :1682-1692)
static std::vector<Edge> inc_aggregation(const Graph& g, const std::vector<Edge>& delta,
                                         const std::vector<u32>& s_pre,
                                         const std::vector<u32>& s_cur,
                                         const std::vector<uint8_t>& refined,
                                         std::vector<u32>& s_pre_next, u32& next_n,
                                         bool changed_only, bool edge_weight_loops) {
  std::vector<Edge> dh;
  for (const Edge& e : delta) dh.push_back({s_pre[e.u], s_pre[e.v], e.w});
  for (u32 v = 0; v < g.n; ++v) {
    if (!refined[v]) continue;
    if (changed_only && s_cur[v] == s_pre[v]) continue;
    double slw = 0.0;
    for (u64 p = g.off[v]; p < g.off[v + 1]; ++p) {
      u32 nb = g.col[p];
      double w = g.w[p];
      if (nb == v) continue;
      bool emit = changed_only
                      ? (s_cur[nb] == s_pre[nb] || !refined[nb] || v < nb)
                      : (s_cur[nb] == s_pre[nb] || v < nb);
      if (emit) {
        dh.push_back({s_pre[v], s_pre[nb], -w});
        dh.push_back({s_cur[v], s_cur[nb], w});
      }
    }
    for (u64 p = g.off[v]; p < g.off[v + 1]; ++p)
      if (g.col[p] == v) slw += g.w[p];
    if (edge_weight_loops) slw = slw / 2.0;
    if (std::fabs(slw) > 1e-12) {
      dh.push_back({s_pre[v], s_pre[v], -slw});
      dh.push_back({s_cur[v], s_cur[v], slw});
    }
  }
  s_pre_next = s_pre;
  for (u32 v = 0; v < g.n; ++v)
    if (refined[v]) s_pre_next[v] = s_cur[v];
  std::vector<Edge> out = compress_sum(dh, 1e-9);
  u32 mx = 0;
  for (u32 x : s_cur) mx = std::max(mx, x);
  for (u32 x : s_pre) mx = std::max(mx, x);
  next_n = mx + 1;
  return out;
}

// hit_leiden.rs:1733-1793 (`def_update`, `propagate_community_assignments`,
// `propagate_changed_nodes_to_prev_level`).
static void def_update(std::vector<std::vector<u32>>& f, const std::vector<std::vector<u32>>& s,
                       std::vector<std::vector<uint8_t>>& changed, u32 P) {
  for (int p = (int)P - 1; p >= 0; --p) {
    if ((u32)p < P - 1) {
      for (size_t v = 0; v < changed[p].size(); ++v)
        if (changed[p][v]) f[p][v] = f[p + 1][s[p][v]];
    }
    if (p > 0) {
      std::vector<uint8_t>& up = changed[p];
      for (size_t v = 0; v < up.size(); ++v) {
        if (!up[v]) continue;
        for (size_t u = 0; u < s[p - 1].size(); ++u)
          if (s[p - 1][u] == v) changed[p - 1][u] = 1;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Hierarchical state (state.rs:19-49) and Algorithm 6 (hit_leiden.rs:936-1018)
// ---------------------------------------------------------------------------
struct State {
  u32 levels = 1;
  std::vector<Graph> sg;  // supergraphs
  std::vector<std::vector<u32>> f, g, s_pre, s_cur;
  std::vector<u32> node_to_comm;
};

static State state_identity(u32 n, u32 levels) {
  State st;
  st.levels = levels;
  std::vector<u32> id(n);
  for (u32 i = 0; i < n; ++i) id[i] = i;
  st.node_to_comm = id;
  for (u32 p = 0; p < levels; ++p) {
    st.f.push_back(id);
    st.g.push_back(id);
    st.s_pre.push_back(id);
    st.s_cur.push_back(id);
  }
  return st;
}

static void grow_map(std::vector<u32>& m, u32 n) {
  while (m.size() < n) m.push_back((u32)m.size());
}

struct HlStats {
  u32 iterations = 0;
  u64 moves = 0, candidates = 0, traversed = 0, splits = 0, merges = 0, changed = 0, refined = 0;
};

static u32 hit_leiden(State& st, u32 delta_n, const std::vector<Edge>& delta, double gamma, int mode,
                      u32 flags, u32 max_rounds, HlStats* stats) {
  const bool keep_loops = flags & OR_FLAG_KEEP_SELF_LOOPS;
  const bool compact = !(flags & OR_FLAG_NO_COMPACT);
  const bool faithful = flags & OR_FLAG_FAITHFUL_SCANS;
  if (st.sg.empty()) st.sg.push_back(graph_from_edges(delta_n, delta));
  u32 P = st.levels;
  std::vector<Edge> cur = delta;
  u32 cur_n = delta_n;
  std::vector<std::vector<uint8_t>> changed(P), refined(P);
  u32 total_it = 0;
  for (u32 p = 0; p < P; ++p) {
    while (st.sg.size() <= p) st.sg.push_back(Graph());
    st.sg[p] = apply_delta(st.sg[p], cur_n, cur, keep_loops);
    u32 np = st.sg[p].n;
    grow_map(st.f[p], np);
    grow_map(st.g[p], np);
    grow_map(st.s_pre[p], np);
    grow_map(st.s_cur[p], np);
    MoveOut mo = inc_movement(st.sg[p], cur, st.f[p], st.s_cur[p], gamma, mode, max_rounds, compact,
                              false, nullptr, (flags & OR_FLAG_HUB_CHECK) ? HUB_CHECK_DEG : 0);
    total_it += mo.iterations;
    RefineOut ro = inc_refinement(st.sg[p], st.f[p], st.s_cur[p], mo.affected, gamma, mode, faithful);
    if (stats) {
      stats->moves += mo.rounds_moves;
      stats->candidates += mo.rounds_candidates;
      stats->traversed += mo.traversed;
      stats->splits += ro.splits;
      stats->merges += ro.merges;
      if (p == 0) {
        for (uint8_t c : mo.changed) stats->changed += c;
        for (uint8_t c : ro.refined) stats->refined += c;
      }
    }
    changed[p] = mo.changed;
    refined[p] = ro.refined;
    if (p + 1 < P) {
      bool any_r = false;
      for (uint8_t c : ro.refined) any_r |= (c != 0);
      if (cur.empty() && !any_r) {  // should_skip_aggregation (:1020-1022)
        cur.clear();
        continue;
      }
      std::vector<u32> sp_next;
      u32 nn = 0;
      std::vector<Edge> nd =
          inc_aggregation(st.sg[p], cur, st.s_pre[p], st.s_cur[p], ro.refined, sp_next, nn,
                          flags & OR_FLAG_AGG_CHANGED_ONLY, flags & OR_FLAG_EDGE_WEIGHT_LOOPS);
      st.s_pre[p] = sp_next;
      cur = nd;
      cur_n = nn;
    }
  }
  // Bitsets are sized by the delta's node count (:952-953); pad to each level.
  for (u32 p = 0; p < P; ++p) {
    changed[p].resize(st.f[p].size(), 0);
    refined[p].resize(st.g[p].size(), 0);
  }
  def_update(st.f, st.s_cur, changed, P);
  def_update(st.g, st.s_cur, refined, P);
  st.node_to_comm = st.g[0];
  if (stats) stats->iterations = total_it;
  return total_it;
}

// ---------------------------------------------------------------------------
// Multi-level extension.  The reference only ever runs one level
// (state.rs:42 sets levels = 1 and nothing raises it), so levels >= 2 are
// defined here, following the spec's Algorithm 1 (bootstrap) and Algorithm 6
// (update) with the changes a consistent hierarchy needs:
//   M1 apply_delta keeps existing self-loops (supernode self-loops carry the
//      intra-sub-community weight);
//   M2 a vertex that moves is always put in K;
//   M3 refinement splits sub-communities into connected components over edges
//      whose ends share both sub-community and community (the Ψ index of
//      Algorithm 2 lines 17-19), so sub-communities stay inside communities;
//   M4 inc-aggregation iterates R ∩ {s_cur != s_pre} and moves a self-loop's
//      edge weight w;
//   M5 after refinement at level p, f^{p+1}(s^p(v)) := f^p(v) for every v;
//   M6 a sub-community id X handed out at level p for a component split from
//      S starts at level p+1 with S's s_pre / s_cur / g values;
//   M7 def-update recomputes f^p = f^{p+1}∘s^p and g^p = g^{p+1}∘s^p top-down
//      for every vertex (g at the top level is the identity);
//   M8 the level-(p+1) nodes created by M6, and those whose community M5
//      changed, join K at level p+1, so that their sub-community is split
//      again when it is no longer connected or no longer inside one community
//      (refined communities stay connected and nested at every level).
// ---------------------------------------------------------------------------
static void ensure_level_size(State& st, u32 p, u32 n) {
  grow_map(st.f[p], n);
  grow_map(st.g[p], n);
  grow_map(st.s_pre[p], n);
  grow_map(st.s_cur[p], n);
  if (st.sg[p].n < n) {
    Graph& g = st.sg[p];
    u64 last = g.off.back();
    g.off.resize((size_t)n + 1, last);
    g.n = n;
  }
}

static u32 hit_leiden_ml(State& st, const std::vector<Edge>& delta, double gamma, int mode,
                         u32 flags, u32 max_rounds, HlStats* stats) {
  const bool compact = !(flags & OR_FLAG_NO_COMPACT);
  const bool faithful = flags & OR_FLAG_FAITHFUL_SCANS;
  u32 P = st.levels;
  std::vector<Edge> cur = delta;
  u32 cur_n = st.sg[0].n;
  u32 total_it = 0;
  std::vector<u32> gained;  // nodes this level gained from splits below (M8)
  for (u32 p = 0; p < P; ++p) {
    st.sg[p] = apply_delta(st.sg[p], std::max(cur_n, st.sg[p].n), cur, true);
    ensure_level_size(st, p, st.sg[p].n);
    MoveOut mo = inc_movement(st.sg[p], cur, st.f[p], st.s_cur[p], gamma, mode, max_rounds,
                              compact, true, &gained,
                              (flags & OR_FLAG_HUB_CHECK) ? HUB_CHECK_DEG : 0);
    total_it += mo.iterations;
    RefineOut ro =
        inc_refinement(st.sg[p], st.f[p], st.s_cur[p], mo.affected, gamma, mode, faithful, true);
    if (stats) {
      stats->moves += mo.rounds_moves;
      stats->candidates += mo.rounds_candidates;
      stats->traversed += mo.traversed;
      stats->splits += ro.splits;
      stats->merges += ro.merges;
      if (p == 0) {
        for (uint8_t c : mo.changed) stats->changed += c;
        for (uint8_t c : ro.refined) stats->refined += c;
      }
    }
    if (std::getenv("HL_ORACLE_TRACE")) {
      u64 nr = 0;
      for (uint8_t c : ro.refined) nr += c;
      std::fprintf(stderr, "level %u n=%u nnz=%llu delta=%zu rounds=%u moves=%llu traversed=%llu "
                   "splits=%llu merges=%llu refined=%llu\n", p, st.sg[p].n,
                   (unsigned long long)st.sg[p].col.size(), cur.size(), mo.iterations,
                   (unsigned long long)mo.rounds_moves, (unsigned long long)mo.traversed,
                   (unsigned long long)ro.splits, (unsigned long long)ro.merges,
                   (unsigned long long)nr);
    }
    if (p + 1 >= P) break;
    // M6: new level-(p+1) nodes inherit the state of the node they split from.
    u32 need = 0;
    for (u32 x : st.s_cur[p]) need = std::max(need, x + 1);
    for (const auto& xo : ro.new_ids) need = std::max(need, xo.first + 1);
    ensure_level_size(st, p + 1, need);
    gained.clear();
    for (const auto& xo : ro.new_ids) {
      st.s_pre[p + 1][xo.first] = st.s_pre[p + 1][xo.second];
      st.s_cur[p + 1][xo.first] = st.s_cur[p + 1][xo.second];
      st.g[p + 1][xo.first] = st.g[p + 1][xo.second];
      gained.push_back(xo.first);
    }
    // M5: project communities up; M8: a node whose community the projection
    // changes joins K at level p+1 as well.
    std::vector<u32> f_before = st.f[p + 1];
    for (u32 v = 0; v < st.sg[p].n; ++v) st.f[p + 1][st.s_cur[p][v]] = st.f[p][v];
    for (u32 x = 0; x < (u32)f_before.size(); ++x)
      if (st.f[p + 1][x] != f_before[x]) gained.push_back(x);
    bool any_r = false;
    for (uint8_t c : ro.refined) any_r |= (c != 0);
    if (cur.empty() && !any_r) {
      cur.clear();
      cur_n = st.sg[p + 1].n;
      continue;
    }
    std::vector<u32> sp_next;
    u32 nn = 0;
    std::vector<Edge> nd = inc_aggregation(st.sg[p], cur, st.s_pre[p], st.s_cur[p], ro.refined,
                                           sp_next, nn, true, true);
    st.s_pre[p] = sp_next;
    cur = nd;
    cur_n = std::max(nn, st.sg[p + 1].n);
  }
  // M7: top-down recompute.
  for (u32 v = 0; v < st.g[P - 1].size(); ++v) st.g[P - 1][v] = v;
  for (int p = (int)P - 2; p >= 0; --p) {
    for (size_t v = 0; v < st.f[p].size(); ++v) {
      st.f[p][v] = st.f[p + 1][st.s_cur[p][v]];
      st.g[p][v] = st.g[p + 1][st.s_cur[p][v]];
    }
  }
  st.node_to_comm = st.g[0];
  if (stats) stats->iterations = total_it;
  return total_it;
}

// Algorithm 1 bootstrap: Move / Refine / Aggregate per level until the
// refinement no longer coarsens (fewer than 1% fewer nodes) or `max_levels`.
static void bootstrap_ml(State& st, u32 n, const std::vector<Edge>& edges, double gamma, int mode,
                         u32 flags, u32 max_rounds, u32 max_levels, HlStats* stats) {
  const bool faithful = flags & OR_FLAG_FAITHFUL_SCANS;
  st = State();
  Graph empty;
  empty.n = n;
  empty.off.assign((size_t)n + 1, 0);
  Graph g0 = apply_delta(empty, n, edges, true);
  st.sg.push_back(g0);
  std::vector<u32> id(n);
  for (u32 i = 0; i < n; ++i) id[i] = i;
  st.f.push_back(id);
  st.g.push_back(id);
  st.s_pre.push_back(id);
  st.s_cur.push_back(id);
  u32 p = 0;
  while (true) {
    Graph& G = st.sg[p];
    u32 np = G.n;
    std::vector<Edge> none;
    MoveOut mo = inc_movement(G, none, st.f[p], st.s_cur[p], gamma, mode, max_rounds, true, true);
    RefineOut ro = inc_refinement(G, st.f[p], st.s_cur[p], mo.affected, gamma, mode, faithful, true);
    if (stats) {
      stats->iterations += mo.iterations;
      stats->moves += mo.rounds_moves;
      stats->traversed += mo.traversed;
      stats->merges += ro.merges;
    }
    // Compact sub-community ids (rank) so that level p+1 has no holes.
    std::vector<u32>& s = st.s_cur[p];
    std::vector<u32> ids(s.begin(), s.end());
    std::sort(ids.begin(), ids.end());
    ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
    for (u32& x : s) x = (u32)(std::lower_bound(ids.begin(), ids.end(), x) - ids.begin());
    st.s_pre[p] = s;
    u32 nn = (u32)ids.size();
    if (p + 1 >= max_levels || nn <= 1 || (u64)nn * 100 >= (u64)np * 99) break;
    // Aggregate G^p by s^p (intra edges become self-loops of weight w).
    std::vector<Edge> recs;
    for (u32 v = 0; v < np; ++v)
      for (u64 q = G.off[v]; q < G.off[v + 1]; ++q) {
        u32 nb = G.col[q];
        if (nb < v) continue;
        // a self-loop appears twice in its row; count it once
        if (nb == v && q + 1 < G.off[v + 1] && G.col[q + 1] == v) continue;
        recs.push_back({s[v], s[nb], G.w[q]});
      }
    std::vector<Edge> agg = compress_sum(recs, -1.0);
    Graph gn;
    gn.n = nn;
    gn.off.assign((size_t)nn + 1, 0);
    st.sg.push_back(apply_delta(gn, nn, agg, true));
    std::vector<u32> fn(nn, 0), idn(nn);
    for (u32 i = 0; i < nn; ++i) idn[i] = i;
    for (u32 v = 0; v < np; ++v) fn[s[v]] = st.f[p][v];
    st.f.push_back(fn);
    st.g.push_back(idn);
    st.s_pre.push_back(idn);
    st.s_cur.push_back(idn);
    ++p;
  }
  st.levels = p + 1;
  u32 P = st.levels;
  for (u32 v = 0; v < st.g[P - 1].size(); ++v) st.g[P - 1][v] = v;
  for (int q = (int)P - 2; q >= 0; --q)
    for (size_t v = 0; v < st.f[q].size(); ++v) {
      st.f[q][v] = st.f[q + 1][st.s_cur[q][v]];
      st.g[q][v] = st.g[q + 1][st.s_cur[q][v]];
    }
  st.node_to_comm = st.g[0];
}

// ---------------------------------------------------------------------------
// Static run(): hit_leiden.rs:30-118 → multilevel_leiden (:167-323).  The
// quality reference for the incremental path (the operation the reference's
// own benchmark times per batch).  thread_rng → seeded splitmix64 shuffle.
// ---------------------------------------------------------------------------
struct SplitMix {
  u64 x;
  u64 next() {
    u64 z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
};

// hit_leiden.rs:776-932 (`single_level_movement`, queue-based branch).
static u32 single_level_movement(const Graph& g, const std::vector<Edge>& dg, std::vector<u32>& f,
                                 double gamma, SplitMix& rng) {
  u32 n = g.n;
  std::vector<uint8_t> active(n, 0);
  for (const Edge& e : dg)
    if (e.w > 0.0 && e.u < n && e.v < n && f[e.u] != f[e.v]) active[e.u] = active[e.v] = 1;
  if (dg.empty()) std::fill(active.begin(), active.end(), 1);
  std::vector<double> k = node_degrees(g);
  double tw = twice_total_weight(k);
  u32 mxf = 0;
  for (u32 x : f) mxf = std::max(mxf, x);
  std::vector<double> d(std::max<size_t>(n, (size_t)mxf + 1), 0.0);
  for (u32 i = 0; i < n; ++i) d[f[i]] += k[i];
  std::vector<u32> qn;
  for (u32 i = 0; i < n; ++i)
    if (active[i]) qn.push_back(i);
  for (size_t i = qn.size(); i > 1; --i) {
    size_t j = rng.next() % i;
    std::swap(qn[i - 1], qn[j]);
  }
  std::deque<u32> q(qn.begin(), qn.end());
  std::vector<uint8_t> inq = active;
  std::vector<double> buf(d.size(), 0.0);
  std::vector<uint8_t> seen(d.size(), 0);
  std::vector<u32> order;
  while (!q.empty()) {
    u32 v = q.front();
    q.pop_front();
    inq[v] = 0;
    u32 cur = f[v];
    u32 best = cur;
    double bestg = 0.0;
    double wcur = 0.0;
    double kv = k[v];
    order.clear();
    for (u64 p = g.off[v]; p < g.off[v + 1]; ++p) {
      u32 nb = g.col[p];
      if (nb == v) continue;
      u32 c = f[nb];
      if (!seen[c]) {
        seen[c] = 1;
        order.push_back(c);
      }
      buf[c] += g.w[p];
      if (c == cur) wcur += g.w[p];
    }
    double dcur = d[cur];
    for (u32 c : order) {
      if (c == cur) continue;
      double gn = move_gain(buf[c], wcur, tw, gamma, kv, dcur, d[c]);
      if (gn > bestg) {
        bestg = gn;
        best = c;
      }
    }
    for (u32 c : order) {
      buf[c] = 0.0;
      seen[c] = 0;
    }
    if (bestg <= 0.0) continue;
    f[v] = best;
    d[cur] -= kv;
    d[best] += kv;
    for (u64 p = g.off[v]; p < g.off[v + 1]; ++p) {
      u32 nb = g.col[p];
      if (nb == v || f[nb] == best || inq[nb]) continue;
      q.push_back(nb);
      inq[nb] = 1;
    }
  }
  return 1;
}

// hit_leiden.rs:676-720.
static double subcommunity_dq_to_empty(const Graph& g, const std::vector<u32>& s,
                                       const std::vector<u32>& f, const std::vector<double>& dS,
                                       u32 S, u32 parent, double gamma, double tw,
                                       const std::vector<double>& k) {
  if (tw == 0.0) return 0.0;
  double ds = S < dS.size() ? dS[S] : 0.0;
  if (ds == 0.0) return 0.0;
  double dpar = 0.0;
  for (u32 i = 0; i < g.n; ++i)
    if (f[i] == parent) dpar += k[i];
  double wsp = 0.0;
  for (u32 i = 0; i < g.n; ++i) {
    if (s[i] != S) continue;
    for (u64 p = g.off[i]; p < g.off[i + 1]; ++p)
      if (f[g.col[p]] == parent) wsp += g.w[p];
  }
  return (0.0 - wsp) / tw + gamma * ds * (dpar - ds) / (tw * tw);
}

// hit_leiden.rs:449-671 (`refine_singleton_merge`).
static std::vector<u32> refine_singleton_merge(const Graph& g, const std::vector<u32>& f,
                                               double gamma) {
  u32 n = g.n;
  if (n == 0) return {};
  std::vector<u32> s = f;
  std::vector<double> k = node_degrees(g);
  double tw = twice_total_weight(k);
  if (tw == 0.0) return s;
  u32 mx = 0;
  for (u32 x : s) mx = std::max(mx, x);
  u64 next_id = (u64)mx + 1;
  std::vector<uint8_t> refined(n, 0);
  std::map<u32, std::vector<u32>> by_sc;
  for (u32 v = 0; v < n; ++v) by_sc[s[v]].push_back(v);
  std::vector<uint8_t> allowed(n, 0), visited(n, 0);
  for (auto& kv : by_sc) {
    const std::vector<u32>& verts = kv.second;
    if (verts.size() <= 1) continue;
    for (u32 v : verts) allowed[v] = 1;
    std::vector<std::vector<u32>> comps;
    for (u32 st : verts) {
      if (visited[st]) continue;
      std::vector<u32> comp;
      std::deque<u32> q{st};
      visited[st] = 1;
      while (!q.empty()) {
        u32 c = q.front();
        q.pop_front();
        comp.push_back(c);
        for (u64 p = g.off[c]; p < g.off[c + 1]; ++p) {
          u32 nb = g.col[p];
          if (allowed[nb] && !visited[nb]) {
            visited[nb] = 1;
            q.push_back(nb);
          }
        }
      }
      comps.push_back(comp);
    }
    for (u32 v : verts) allowed[v] = visited[v] = 0;
    if (comps.size() <= 1) continue;
    // Largest; on equal sizes the smallest minimum node id (:507-518).
    size_t keep = 0;
    for (size_t i = 1; i < comps.size(); ++i) {
      u32 mi = *std::min_element(comps[i].begin(), comps[i].end());
      u32 mk = *std::min_element(comps[keep].begin(), comps[keep].end());
      if (comps[i].size() > comps[keep].size() ||
          (comps[i].size() == comps[keep].size() && mi < mk))
        keep = i;
    }
    for (size_t i = 0; i < comps.size(); ++i) {
      if (i == keep) continue;
      u32 nid = (u32)next_id++;
      for (u32 v : comps[i]) {
        s[v] = nid;
        refined[v] = 1;
      }
    }
  }
  u32 smax = 0;
  for (u32 x : s) smax = std::max(smax, x);
  std::vector<u64> sizes((size_t)smax + 1, 0);
  std::vector<double> dS((size_t)smax + 1, 0.0);
  for (u32 v = 0; v < n; ++v) {
    sizes[s[v]] += 1;
    dS[s[v]] += k[v];
  }
  std::vector<u32> rs;
  for (u32 v = 0; v < n; ++v)
    if (refined[v]) rs.push_back(v);
  std::stable_sort(rs.begin(), rs.end(), [&](u32 a, u32 b) { return k[a] < k[b]; });
  const double EPS = 1e-12;
  std::map<u32, double> nsc;
  for (u32 v : rs) {
    u32 cs = s[v];
    if (sizes[cs] != 1) continue;
    u32 pc = f[v];
    double kv = k[v];
    nsc.clear();
    double wcur = 0.0;
    for (u64 p = g.off[v]; p < g.off[v + 1]; ++p) {
      u32 nb = g.col[p];
      if (nb == v) continue;
      if (f[nb] != pc) continue;
      nsc[s[nb]] += g.w[p];
      if (s[nb] == cs) wcur += g.w[p];
    }
    if (nsc.empty()) continue;
    std::vector<u32> filtered;
    for (auto& kv2 : nsc) {
      u32 c = kv2.first;
      if (c == cs) continue;
      double dq = subcommunity_dq_to_empty(g, s, f, dS, c, pc, gamma, tw, k);
      if (dq <= EPS) filtered.push_back(c);
    }
    if (filtered.empty()) continue;
    u32 best = cs;
    double bestg = 0.0, bestw = -1.0;
    for (u32 c : filtered) {
      double wc = nsc[c];
      double dcs = dS[cs];
      double dc = dS[c];
      double gn = (wc - wcur) / tw + gamma * kv * (dcs - kv - dc) / (tw * tw);
      bool better = (gn > bestg + EPS) ||
                    (std::fabs(gn - bestg) <= EPS &&
                     (wc > bestw + EPS || (std::fabs(wc - bestw) <= EPS && c < best)));
      if (better) {
        bestg = gn;
        best = c;
        bestw = wc;
      }
    }
    if (bestg > EPS) {
      s[v] = best;
      sizes[cs] = sizes[cs] ? sizes[cs] - 1 : 0;
      sizes[best] += 1;
      dS[cs] -= kv;
      dS[best] += kv;
    }
  }
  return s;
}

// hit_leiden.rs:726-773 (`aggregate_graph`), canonical edge order.
static std::vector<Edge> aggregate_graph(const std::vector<Edge>& edges, const std::vector<u32>& part,
                                         std::unordered_map<u32, u32>& remap, u32& nn) {
  remap.clear();
  u32 next = 0;
  for (u32 c : part)
    if (!remap.count(c)) remap[c] = next++;
  std::map<std::pair<u32, u32>, double> em;
  for (const Edge& e : edges) {
    u32 cu = remap[part[e.u]], cv = remap[part[e.v]];
    std::pair<u32, u32> key = cu <= cv ? std::make_pair(cu, cv) : std::make_pair(cv, cu);
    em[key] += e.w;
  }
  std::vector<Edge> out;
  for (auto& kv : em) out.push_back({kv.first.first, kv.first.second, kv.second});
  nn = next;
  return out;
}

struct RunOut {
  std::vector<u32> part;
  std::vector<std::vector<u32>> hierarchy;
  u32 iterations = 0;
  double quality = 0.0;
};

static RunOut run_multilevel(u32 n, const std::vector<Edge>& edges, double gamma, u32 max_levels,
                             u64 seed) {
  SplitMix rng{seed};
  RunOut out;
  Graph g0 = graph_from_edges(n, edges);
  std::vector<u32> f(n), id(n);
  for (u32 i = 0; i < n; ++i) f[i] = id[i] = i;
  out.iterations += single_level_movement(g0, edges, f, gamma, rng);
  std::vector<u32> sub = refine_singleton_merge(g0, f, gamma);
  std::vector<u32> node_to_comm = f;
  {
    std::vector<u32> c = node_to_comm;
    canonicalize(c);
    out.hierarchy.push_back(c);
  }
  size_t prev = count_unique(node_to_comm);
  for (u32 level = 1; level < max_levels; ++level) {
    size_t cur_sub = count_unique(sub);
    if (cur_sub <= 1) break;
    std::unordered_map<u32, u32> remap;
    u32 cn = 0;
    std::vector<Edge> coarse = aggregate_graph(edges, sub, remap, cn);
    if (cn <= 1 || coarse.empty()) break;
    // build_coarse_initial_partition (:325-345), ascending sub-community id.
    std::map<u32, u32> sub_to_comm;
    for (u32 i = 0; i < n; ++i)
      if (!sub_to_comm.count(sub[i])) sub_to_comm[sub[i]] = node_to_comm[i];
    std::unordered_map<u32, u32> cremap;
    u32 nextc = 0;
    std::vector<u32> cf(cn, 0);
    for (auto& kv : sub_to_comm) {
      auto it = remap.find(kv.first);
      if (it == remap.end()) continue;
      auto jt = cremap.find(kv.second);
      if (jt == cremap.end()) jt = cremap.emplace(kv.second, nextc++).first;
      cf[it->second] = jt->second;
    }
    Graph cg = graph_from_edges(cn, coarse);
    out.iterations += single_level_movement(cg, coarse, cf, gamma, rng);
    for (u32& c : sub) c = cf[remap[c]];
    node_to_comm = sub;
    f = node_to_comm;
    {
      std::vector<u32> c = node_to_comm;
      canonicalize(c);
      out.hierarchy.push_back(c);
    }
    size_t nc = count_unique(node_to_comm);
    sub = refine_singleton_merge(g0, node_to_comm, gamma);
    if (nc >= prev) break;
    prev = nc;
  }
  f = node_to_comm;
  out.iterations += single_level_movement(g0, edges, f, gamma, rng);
  node_to_comm = f;
  std::vector<u32> fin = node_to_comm;
  canonicalize(fin);
  if (out.hierarchy.empty() || out.hierarchy.back() != fin) out.hierarchy.push_back(fin);
  canonicalize(node_to_comm);
  out.part = node_to_comm;
  out.quality = modularity_edges(n, edges, out.part.data());
  return out;
}

}  // namespace ora

// ===========================================================================
// C ABI used by the test harness (ctypes).  Plain arrays in and out.
// ===========================================================================
using namespace ora;

struct or_graph {
  Graph g;
};
struct or_state {
  State st;
  double gamma = 1.0;
  int mode = OR_MODE_THROUGHPUT;
  u32 flags = 0;
  u32 max_rounds = 20;
};

static std::vector<Edge> make_edges(const uint32_t* src, const uint32_t* dst, const double* w,
                                    uint64_t m) {
  std::vector<Edge> e(m);
  for (uint64_t i = 0; i < m; ++i) e[i] = {src[i], dst[i], w ? w[i] : 1.0};
  return e;
}

extern "C" {

or_graph* or_graph_from_edges(uint32_t n, const uint32_t* src, const uint32_t* dst, const double* w,
                              uint64_t m) {
  for (uint64_t i = 0; i < m; ++i)
    if (src[i] >= n || dst[i] >= n) return nullptr;
  or_graph* G = new or_graph;
  G->g = graph_from_edges(n, make_edges(src, dst, w, m));
  return G;
}

void or_graph_free(or_graph* G) { delete G; }

uint32_t or_graph_nodes(const or_graph* G) { return G->g.n; }
uint64_t or_graph_entries(const or_graph* G) { return G->g.col.size(); }

void or_graph_csr(const or_graph* G, uint64_t* off, uint32_t* col, double* w) {
  const Graph& g = G->g;
  if (off) std::memcpy(off, g.off.data(), sizeof(uint64_t) * (g.n + 1));
  if (col) std::memcpy(col, g.col.data(), sizeof(uint32_t) * g.col.size());
  if (w) std::memcpy(w, g.w.data(), sizeof(double) * g.w.size());
}

or_graph* or_graph_apply_delta(const or_graph* G, uint32_t delta_n, const uint32_t* src,
                               const uint32_t* dst, const double* w, uint64_t k, int keep_loops) {
  or_graph* R = new or_graph;
  R->g = apply_delta(G->g, delta_n, make_edges(src, dst, w, k), keep_loops != 0);
  return R;
}

void or_node_degrees(const or_graph* G, double* out) {
  std::vector<double> k = node_degrees(G->g);
  std::memcpy(out, k.data(), sizeof(double) * k.size());
}

double or_twice_total_weight(const or_graph* G) { return twice_total_weight(node_degrees(G->g)); }

double or_tree_sum(const double* x, uint64_t n) {
  return tree_sum(std::vector<double>(x, x + n));
}

double or_modularity_edges(uint32_t n, const uint32_t* src, const uint32_t* dst, const double* w,
                           uint64_t m, const uint32_t* part) {
  return modularity_edges(n, make_edges(src, dst, w, m), part);
}

double or_modularity_csr(const or_graph* G, const uint32_t* part) {
  return modularity_csr(G->g, part);
}

void or_canonicalize(uint32_t* c, uint64_t n) {
  std::vector<u32> v(c, c + n);
  canonicalize(v);
  std::memcpy(c, v.data(), sizeof(u32) * n);
}

int or_num_threads(void) { return ora::num_threads(); }

void or_set_num_threads(int t) { ora::g_threads.store(t > 0 ? t : 0); }

uint64_t or_select_decoupled(const uint32_t* node, const uint32_t* from, const uint32_t* to,
                             const double* kdeg, const double* gain, uint64_t m,
                             uint32_t* out_nodes) {
  std::vector<Move> c(m);
  for (uint64_t i = 0; i < m; ++i) c[i] = {node[i], from[i], to[i], kdeg ? kdeg[i] : 1.0, gain[i]};
  std::vector<Move> sel = select_decoupled(c);
  for (size_t i = 0; i < sel.size(); ++i) out_nodes[i] = sel[i].node;
  return sel.size();
}

void or_move_eval(const or_graph* G, const uint32_t* f, const double* d, uint64_t d_len,
                  const double* k, double tw, double gamma, const uint32_t* verts, uint64_t nv,
                  uint32_t* out_to, double* out_gain) {
  const Graph& g = G->g;
  std::vector<u32> fv(f, f + g.n);
  std::vector<double> dv(d, d + d_len), kv(k, k + g.n);
  MoveScratch sc;
  sc.buf.assign(d_len + g.n + 1, 0.0);
  for (uint64_t i = 0; i < nv; ++i) {
    Eval e = eval_move(g, verts[i], fv, dv, kv, tw, gamma, true, sc);
    out_to[i] = e.to;
    out_gain[i] = e.gain;
  }
}

uint32_t or_inc_movement(const or_graph* G, const uint32_t* dsrc, const uint32_t* ddst,
                         const double* dw, uint64_t dk, uint32_t* f, const uint32_t* s,
                         double gamma, int mode, uint32_t max_rounds, int compact, int mark_moved,
                         uint8_t* out_changed, uint8_t* out_affected) {
  const Graph& g = G->g;
  std::vector<u32> fv(f, f + g.n), sv(s, s + g.n);
  MoveOut mo = inc_movement(g, make_edges(dsrc, ddst, dw, dk), fv, sv, gamma, mode, max_rounds,
                            compact != 0, mark_moved != 0);
  std::memcpy(f, fv.data(), sizeof(u32) * g.n);
  if (out_changed) std::memcpy(out_changed, mo.changed.data(), g.n);
  if (out_affected) std::memcpy(out_affected, mo.affected.data(), g.n);
  return mo.iterations;
}

void or_inc_refinement(const or_graph* G, const uint32_t* f, uint32_t* s, const uint8_t* affected,
                       double gamma, int mode, int faithful, int cc_same_community,
                       uint8_t* out_refined) {
  const Graph& g = G->g;
  std::vector<u32> fv(f, f + g.n), sv(s, s + g.n);
  std::vector<uint8_t> av(affected, affected + g.n);
  RefineOut ro = inc_refinement(g, fv, sv, av, gamma, mode, faithful != 0, cc_same_community != 0);
  std::memcpy(s, sv.data(), sizeof(u32) * g.n);
  if (out_refined) std::memcpy(out_refined, ro.refined.data(), g.n);
}

// Returns the number of compressed ΔH edges; writes up to `cap` of them.
uint64_t or_inc_aggregation(const or_graph* G, const uint32_t* dsrc, const uint32_t* ddst,
                            const double* dw, uint64_t dk, const uint32_t* s_pre,
                            const uint32_t* s_cur, const uint8_t* refined, uint32_t flags,
                            uint32_t* out_s_pre, uint32_t* out_next_n, uint32_t* out_u,
                            uint32_t* out_v, double* out_w, uint64_t cap) {
  const Graph& g = G->g;
  std::vector<u32> sp(s_pre, s_pre + g.n), sc(s_cur, s_cur + g.n), nsp;
  std::vector<uint8_t> rv(refined, refined + g.n);
  u32 nn = 0;
  std::vector<Edge> out = inc_aggregation(g, make_edges(dsrc, ddst, dw, dk), sp, sc, rv, nsp, nn,
                                          flags & OR_FLAG_AGG_CHANGED_ONLY,
                                          flags & OR_FLAG_EDGE_WEIGHT_LOOPS);
  if (out_s_pre) std::memcpy(out_s_pre, nsp.data(), sizeof(u32) * g.n);
  if (out_next_n) *out_next_n = nn;
  for (size_t i = 0; i < out.size() && i < cap; ++i) {
    out_u[i] = out[i].u;
    out_v[i] = out[i].v;
    out_w[i] = out[i].w;
  }
  return out.size();
}

// def_update over P levels given as concatenated arrays; sizes[p] = n_p.
void or_def_update(uint32_t P, const uint32_t* sizes, uint32_t* f_cat, const uint32_t* s_cat,
                   uint8_t* changed_cat) {
  std::vector<std::vector<u32>> f(P), s(P);
  std::vector<std::vector<uint8_t>> ch(P);
  uint64_t o = 0;
  for (u32 p = 0; p < P; ++p) {
    f[p].assign(f_cat + o, f_cat + o + sizes[p]);
    s[p].assign(s_cat + o, s_cat + o + sizes[p]);
    ch[p].assign(changed_cat + o, changed_cat + o + sizes[p]);
    o += sizes[p];
  }
  def_update(f, s, ch, P);
  o = 0;
  for (u32 p = 0; p < P; ++p) {
    std::memcpy(f_cat + o, f[p].data(), sizeof(u32) * sizes[p]);
    std::memcpy(changed_cat + o, ch[p].data(), sizes[p]);
    o += sizes[p];
  }
}

or_state* or_state_new(uint32_t n, uint32_t levels, double gamma, int mode, uint32_t flags,
                       uint32_t max_rounds) {
  or_state* S = new or_state;
  S->st = state_identity(n, levels ? levels : 1);
  S->gamma = gamma;
  S->mode = mode;
  S->flags = flags;
  S->max_rounds = max_rounds ? max_rounds : 20;
  return S;
}

void or_state_free(or_state* S) { delete S; }

// Push an empty level-0 supergraph of n nodes (the reference tests' pattern,
// hit_leiden.rs:3119-3124) so that the first call does not double weights.
void or_state_push_empty_graph(or_state* S, uint32_t n) {
  Graph g;
  g.n = n;
  g.off.assign((size_t)n + 1, 0);
  S->st.sg.push_back(g);
}

int or_hit_leiden(or_state* S, uint32_t delta_n, const uint32_t* src, const uint32_t* dst,
                  const double* w, uint64_t k, or_stats* stats) {
  HlStats hs;
  if (S->flags & OR_FLAG_MULTILEVEL)
    hit_leiden_ml(S->st, make_edges(src, dst, w, k), S->gamma, S->mode, S->flags, S->max_rounds,
                  &hs);
  else
    hit_leiden(S->st, delta_n, make_edges(src, dst, w, k), S->gamma, S->mode, S->flags,
               S->max_rounds, &hs);
  if (stats) {
    stats->iterations = hs.iterations;
    stats->moves = hs.moves;
    stats->candidates = hs.candidates;
    stats->traversed = hs.traversed;
    stats->splits = hs.splits;
    stats->merges = hs.merges;
    stats->changed = hs.changed;
    stats->refined = hs.refined;
  }
  return 0;
}

uint32_t or_state_levels(const or_state* S) { return S->st.levels; }

// Replace the state by `levels` levels imported level by level (used to start
// the CPU baseline from an already bootstrapped state).
void or_state_import_begin(or_state* S, uint32_t levels, uint32_t flags) {
  S->st = State();
  S->st.levels = levels;
  S->st.sg.resize(levels);
  S->st.f.resize(levels);
  S->st.g.resize(levels);
  S->st.s_pre.resize(levels);
  S->st.s_cur.resize(levels);
  S->flags = flags;
}

int or_state_import_level(or_state* S, uint32_t level, uint32_t n, const uint64_t* off,
                          const uint32_t* col, const double* w, const uint32_t* f,
                          const uint32_t* g, const uint32_t* s_pre, const uint32_t* s_cur) {
  State& st = S->st;
  if (level >= st.levels) return -1;
  Graph& G = st.sg[level];
  G.n = n;
  G.off.assign(off, off + (size_t)n + 1);
  G.col.assign(col, col + off[n]);
  G.w.assign(w, w + off[n]);
  st.f[level].assign(f, f + n);
  st.g[level].assign(g, g + n);
  st.s_pre[level].assign(s_pre, s_pre + n);
  st.s_cur[level].assign(s_cur, s_cur + n);
  if (level == 0) st.node_to_comm = st.g[0];
  return 0;
}

int or_state_bootstrap(or_state* S, uint32_t n, const uint32_t* src, const uint32_t* dst,
                       const double* w, uint64_t m, uint32_t max_levels, or_stats* stats) {
  HlStats hs;
  bootstrap_ml(S->st, n, make_edges(src, dst, w, m), S->gamma, S->mode, S->flags, S->max_rounds,
               max_levels ? max_levels : 10, &hs);
  S->flags |= OR_FLAG_MULTILEVEL;
  if (stats) {
    stats->iterations = hs.iterations;
    stats->moves = hs.moves;
    stats->traversed = hs.traversed;
    stats->merges = hs.merges;
  }
  return 0;
}

uint32_t or_state_level_nodes(const or_state* S, uint32_t level, int which) {
  const State& st = S->st;
  if (level >= st.levels) return 0;
  switch (which) {
    case OR_MAP_F: return (uint32_t)st.f[level].size();
    case OR_MAP_G: return (uint32_t)st.g[level].size();
    case OR_MAP_S_PRE: return (uint32_t)st.s_pre[level].size();
    case OR_MAP_S_CUR: return (uint32_t)st.s_cur[level].size();
    case OR_MAP_NODE_TO_COMM: return (uint32_t)st.node_to_comm.size();
  }
  return 0;
}

int or_state_get_map(const or_state* S, uint32_t level, int which, uint32_t* out) {
  const State& st = S->st;
  if (which == OR_MAP_NODE_TO_COMM) {
    std::memcpy(out, st.node_to_comm.data(), sizeof(u32) * st.node_to_comm.size());
    return 0;
  }
  if (level >= st.levels) return -1;
  const std::vector<u32>* m = nullptr;
  switch (which) {
    case OR_MAP_F: m = &st.f[level]; break;
    case OR_MAP_G: m = &st.g[level]; break;
    case OR_MAP_S_PRE: m = &st.s_pre[level]; break;
    case OR_MAP_S_CUR: m = &st.s_cur[level]; break;
    default: return -1;
  }
  std::memcpy(out, m->data(), sizeof(u32) * m->size());
  return 0;
}

int or_state_set_map(or_state* S, uint32_t level, int which, const uint32_t* in, uint32_t n) {
  State& st = S->st;
  if (level >= st.levels) return -1;
  std::vector<u32>* m = nullptr;
  switch (which) {
    case OR_MAP_F: m = &st.f[level]; break;
    case OR_MAP_G: m = &st.g[level]; break;
    case OR_MAP_S_PRE: m = &st.s_pre[level]; break;
    case OR_MAP_S_CUR: m = &st.s_cur[level]; break;
    default: return -1;
  }
  m->assign(in, in + n);
  return 0;
}

const or_graph* or_state_graph(or_state* S, uint32_t level) {
  if (level >= S->st.sg.size()) return nullptr;
  return reinterpret_cast<const or_graph*>(&S->st.sg[level]);
}

double or_state_modularity(const or_state* S, uint32_t level, int which) {
  const State& st = S->st;
  if (level >= st.sg.size()) return 0.0;
  const std::vector<u32>* m = which == OR_MAP_S_CUR ? &st.s_cur[level] : &st.f[level];
  return modularity_csr(st.sg[level], m->data());
}

double or_run(uint32_t n, const uint32_t* src, const uint32_t* dst, const double* w, uint64_t m,
              double gamma, uint32_t max_levels, uint64_t seed, uint32_t* out_part,
              uint32_t* out_levels) {
  RunOut ro = run_multilevel(n, make_edges(src, dst, w, m), gamma, max_levels, seed);
  if (out_part) std::memcpy(out_part, ro.part.data(), sizeof(u32) * n);
  if (out_levels) *out_levels = (uint32_t)ro.hierarchy.size();
  return ro.quality;
}

int or_hub_check_selftest(void) { return ora::hub_check_selftest(); }

void or_hub_check_counters(uint64_t out[6]) {
  for (int i = 0; i < 6; ++i) out[i] = ora::g_hub_check[i].exchange(0);
}

}  // extern "C"
