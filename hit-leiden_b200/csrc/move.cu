// move.cu — inc-movement, throughput mode (hit_leiden.rs:1024-1101 →
// throughput.rs:80-236 → parallel_frontier.rs:133-239).
//
// Per round, on a snapshot of f and d(C):
//   1. every active vertex finds its best move (warp per vertex; neighbour
//      communities accumulated in first-encounter CSR order so ties go to the
//      earliest candidate, exactly like the reference's dirty list + strict >);
//   2. positive candidates are sorted by (gain desc, node asc);
//   3. the reference's sequential greedy "no move may leave an acceptor or
//      enter an emitter" selection is reproduced exactly with deterministic
//      reservations: a candidate is decided once it holds the minimum rank on
//      every endpoint community whose role is still open;
//   4. accepted moves are applied, d(C) updated in selected order, and the
//      next frontier / K set marked.
#include <cstring>

#include "hl_engine.cuh"

namespace hl {

static inline u32 grid_for(u64 n, u32 block = 256) {
  u64 g = (n + block - 1) / block;
  if (g > 148u * 64u) g = 148u * 64u;
  return g ? (u32)g : 1u;
}

// ----------------------------------------------------------------------------
// Seeding: inc_movement lines 2-8 (hit_leiden.rs:1037-1057).
// ----------------------------------------------------------------------------
// M8 of the multi-level extension: the K marks the level below handed up.
__global__ void k_or_flags(const u8* src, u32 n, u8* dst) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    if (src[i]) dst[i] = 1;
}

__global__ void k_seed(const u32* u, const u32* v, const double* w, u64 k, const u32* f,
                       const u32* s, u8* active, u8* affected) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < k; i += (u64)gridDim.x * blockDim.x) {
    u32 a = u[i], b = v[i];
    double al = w ? w[i] : 1.0;
    bool same_f = f[a] == f[b];
    if ((al > 0.0 && !same_f) || (al < 0.0 && same_f)) {
      active[a] = 1;
      active[b] = 1;
    }
    if (s[a] == s[b]) {
      affected[a] = 1;
      affected[b] = 1;
    }
  }
}

// ----------------------------------------------------------------------------
// Community degrees d(C) = Σ_{f(v)=C} k_v (hit_leiden.rs:1060-1066).
// ----------------------------------------------------------------------------
__global__ void k_comm_deg_atomic(u32 n, const u32* part, const double* k, double* d) {
  __shared__ double sk[256];
  __shared__ u32 sc[256];
  const u32 lane = threadIdx.x & 31;
  const u32 wbase = threadIdx.x & ~31u;
  for (u64 base = blockIdx.x * (u64)blockDim.x; base < n; base += (u64)gridDim.x * blockDim.x) {
    u64 v = base + threadIdx.x;
    bool ok = v < n;
    u32 c = ok ? part[v] : NONE32;
    double kv = ok ? k[v] : 0.0;
    sk[threadIdx.x] = kv;
    sc[threadIdx.x] = c;
    __syncwarp();
    u32 grp = __match_any_sync(0xffffffffu, c);
    if (ok && lane == (u32)(__ffs(grp) - 1)) {
      double s = 0.0;
      for (u32 m = grp; m; m &= m - 1) s += sk[wbase + __ffs(m) - 1];
      atomicAdd(&d[c], s);
    }
    __syncwarp();
  }
}

// Ordered variant: nodes sorted by (community, node), their degrees gathered
// into that order (vals); one warp per community sums its members' degrees in
// ascending node order.  The number of communities is read on the device
// (exclusive scan of the segment heads at the last position plus the last
// head).  Communities of RUN_FOLD_MIN or more members are listed for
// k_comm_deg_runs.
__global__ void k_comm_deg_ordered(const u32* seg_last, const u32* head_last, const u32* ukeys,
                                   const u32* ustart, u32 n, const double* vals, double* d,
                                   u32* longl, u32* longn) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  const u32 nu = *seg_last + *head_last;
  for (u64 j = warp; j < nu; j += nwarps) {
    u32 a = ustart[j], b = (j + 1 < nu) ? ustart[j + 1] : n;
    if (b - a >= RUN_FOLD_MIN) {
      fold_defer(longl, longn, (u32)j);
      continue;
    }
    double s = warp_ordered_sum(a, b, 0.0, [&](u64 t) { return vals[t]; },
                                [](u64) { return true; });
    if (lane == 0) d[ukeys[j]] = s;
  }
}

// The large communities listed by k_comm_deg_ordered, folded in runs (the
// same bits).
__global__ void k_comm_deg_runs(const u32* longl, const u32* longn, const u32* seg_last,
                                const u32* head_last, const u32* ukeys, const u32* ustart, u32 n,
                                const double* vals, double* d) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  const u32 nu = *seg_last + *head_last;
  const u32 nl = *longn;
  for (u64 i = warp; i < nl; i += nwarps) {
    const u32 j = longl[i];
    u32 a = ustart[j], b = (j + 1 < nu) ? ustart[j + 1] : n;
    double s = warp_fold_runs(a, b, 0.0, vals);
    if (lane == 0) d[ukeys[j]] = s;
  }
}

// out[t] = src[idx[t]]: the terms of an ordered sum gathered into sum order.
__global__ void k_gather_f64(const u32* idx, const double* src, u64 n, double* out) {
  for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < n; t += (u64)gridDim.x * blockDim.x)
    out[t] = src[idx[t]];
}

__global__ void k_copy_u32(const u32* a, u32* b, u64 n) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    b[i] = a[i];
}

__global__ void k_heads_u32(const u32* sk, u64 n, u32* head) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    head[i] = (i == 0 || sk[i] != sk[i - 1]) ? 1u : 0u;
}

__global__ void k_seg_compact(const u32* head, const u32* segid, const u32* sk, u64 n,
                              u32* ukeys, u32* ustart) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    if (head[i]) {
      ukeys[segid[i]] = sk[i];
      ustart[segid[i]] = (u32)i;
    }
}

// d[c] for every c in [0, ncomm_cap): zeroed, then filled from `part`.
static void recompute_comm_degrees_impl(Engine& E, Level& L, const u32* part, u32 ncomm_cap,
                                        double* d);

void recompute_comm_degrees(Engine& E, Level& L, const u32* part, u32 ncomm_cap, double* d) {
  cudaEvent_t ev = E.kt_begin();
  recompute_comm_degrees_impl(E, L, part, ncomm_cap, d);
  E.kt_end(KT_COMM_DEG, ev);
}

static void recompute_comm_degrees_impl(Engine& E, Level& L, const u32* part, u32 ncomm_cap,
                                        double* d) {
  cudaStream_t st = E.stream;
  u32 n = L.g.n;
  HL_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * (size_t)ncomm_cap, st));
  if (!n) return;
  if (E.integral) {
    ++E.nlaunch, k_comm_deg_atomic<<<grid_for(n), 256, 0, st>>>(n, part, L.k.p, d);
    HL_LAUNCH_CHECK();
    return;
  }
  Scratch& S = E.sc;
  S.order.ensure(E.mem, n);
  S.order2.ensure(E.mem, n);
  S.used.ensure(E.mem, n);
  S.rank.ensure(E.mem, n);
  S.cand_node.ensure(E.mem, n);
  S.sel_node.ensure(E.mem, n);
  S.segid.ensure(E.mem, n);
  ++E.nlaunch, k_iota<<<grid_for(n), 256, 0, st>>>(S.order.p, n);
  ++E.nlaunch, k_copy_u32<<<grid_for(n), 256, 0, st>>>(part, S.used.p, n);
  HL_LAUNCH_CHECK();
  u32* kin = S.used.p;
  u32* kout = S.rank.p;
  u32* vin = S.order.p;
  u32* vout = S.order2.p;
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceRadixSort::SortPairs(t, b, kin, kout, vin, vout, (int64_t)n, 0,
                                           bits_for(ncomm_cap ? ncomm_cap - 1 : 0), st);
  });
  ++E.nlaunch, k_heads_u32<<<grid_for(n), 256, 0, st>>>(kout, n, S.cand_node.p);
  HL_LAUNCH_CHECK();
  u32* h = S.cand_node.p;
  u32* sid = S.segid.p;
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceScan::ExclusiveSum(t, b, h, sid, (int64_t)n, st);
  });
  ++E.nlaunch, k_seg_compact<<<grid_for(n), 256, 0, st>>>(h, sid, kout, n, S.used.p, S.sel_node.p);
  S.fvals.ensure(E.mem, n);
  ++E.nlaunch, k_gather_f64<<<grid_for(n), 256, 0, st>>>(vout, L.k.p, n, S.fvals.p);
  FoldList fl = fold_list(E, n, n);
  ++E.nlaunch, k_comm_deg_ordered<<<grid_for((u64)n * 32), 256, 0, st>>>(
      sid + n - 1, h + n - 1, S.used.p, S.sel_node.p, n, S.fvals.p, d, fl.seg, fl.cnt);
  ++E.nlaunch, k_comm_deg_runs<<<FOLD_BLOCKS, 256, 0, st>>>(
      fl.seg, fl.cnt, sid + n - 1, h + n - 1, S.used.p, S.sel_node.p, n, S.fvals.p, d);
  HL_LAUNCH_CHECK();
}

// ----------------------------------------------------------------------------
// Label compaction by rank when some id reached >= limit.
// ----------------------------------------------------------------------------
__global__ void k_mark_used(const u32* lab, u32 n, u32* used) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    used[lab[i]] = 1;
}
__global__ void k_relabel(u32* lab, u32 n, const u32* rank) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    lab[i] = rank[lab[i]];
}

// Rank-compacts labels in place; returns the number of distinct labels.
u32 rank_compact(Engine& E, u32* labels, u32 n, u32 id_bound) {
  cudaStream_t st = E.stream;
  Scratch& S = E.sc;
  // One extra (zero) slot so that the exclusive scan's last entry is the
  // number of distinct labels.
  const size_t len = (size_t)id_bound + 2;
  S.used.ensure(E.mem, len);
  S.rank.ensure(E.mem, len);
  HL_CUDA(cudaMemsetAsync(S.used.p, 0, sizeof(u32) * len, st));
  ++E.nlaunch, k_mark_used<<<grid_for(n), 256, 0, st>>>(labels, n, S.used.p);
  HL_LAUNCH_CHECK();
  u32* a = S.used.p;
  u32* r = S.rank.p;
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceScan::ExclusiveSum(t, b, a, r, (int64_t)len, st);
  });
  u32 distinct = E.read_u32(r + id_bound + 1);
  ++E.nlaunch, k_relabel<<<grid_for(n), 256, 0, st>>>(labels, n, S.rank.p);
  HL_LAUNCH_CHECK();
  return distinct;
}

static u32 max_label(Engine& E, const u32* labels, u32 n) {
  if (!n) return 0;
  u32* out = E.sc.cnt.p + 12;
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceReduce::Max(t, b, labels, out, (int64_t)n, E.stream);
  });
  return E.read_u32(out);
}

void compact_labels_if_needed(Engine& E, u32* labels, u32 n, u32 limit) {
  if (!n) return;
  E.sc.cnt.ensure(E.mem, 16);
  u32 mx = max_label(E, labels, n);
  if (mx < limit) return;
  rank_compact(E, labels, n, mx);
}

enum EvalKind { EVAL_MOVE = 0, EVAL_REFINE = 1 };

// ----------------------------------------------------------------------------
// Decoupled selection (throughput.rs:204-236) by deterministic reservations.
// ----------------------------------------------------------------------------
enum : u32 { ROLE_EMIT = 1, ROLE_ACC = 2 };
enum : u8 { ST_UNDECIDED = 0, ST_ACCEPTED = 1, ST_REJECTED = 2 };

__device__ __forceinline__ u32 role_bits(u32 r, u32 round) { return (r >> 2) == round ? (r & 3u) : 0u; }

__global__ void k_reserve(u32 M, const u32* from, const u32* to, u8* status, u8* nmask,
                          const u32* role, unsigned long long* res, u32 round, u64 e) {
  for (u64 r = blockIdx.x * (u64)blockDim.x + threadIdx.x; r < M; r += (u64)gridDim.x * blockDim.x) {
    if (status[r] != ST_UNDECIDED) continue;
    u32 A = from[r], B = to[r];
    u32 ba = role_bits(role[A], round), bb = role_bits(role[B], round);
    if ((ba & ROLE_ACC) || (bb & ROLE_EMIT)) {
      status[r] = ST_REJECTED;
      continue;
    }
    unsigned long long key = ((unsigned long long)e << 32) | (unsigned long long)(0xFFFFFFFFu - (u32)r);
    u8 m = 0;
    if (ba == 0) {
      m |= 1;
      atomicMax(&res[A], key);
    }
    if (bb == 0) {
      m |= 2;
      atomicMax(&res[B], key);
    }
    nmask[r] = m;
  }
}

__global__ void k_decide(u32 M, const u32* from, const u32* to, u8* status, const u8* nmask,
                         u32* role, const unsigned long long* res, u32 round, u64 e,
                         u32* undecided) {
  u32 local = 0;
  for (u64 r = blockIdx.x * (u64)blockDim.x + threadIdx.x; r < M; r += (u64)gridDim.x * blockDim.x) {
    if (status[r] != ST_UNDECIDED) continue;
    u32 A = from[r], B = to[r];
    u8 m = nmask[r];
    unsigned long long key = ((unsigned long long)e << 32) | (unsigned long long)(0xFFFFFFFFu - (u32)r);
    bool ok = (!(m & 1) || res[A] == key) && (!(m & 2) || res[B] == key);
    if (!ok) {
      ++local;
      continue;
    }
    status[r] = ST_ACCEPTED;
    if (A == B) {
      role[A] = (round << 2) | ROLE_EMIT | ROLE_ACC;
    } else {
      role[A] = (round << 2) | ROLE_EMIT;
      role[B] = (round << 2) | ROLE_ACC;
    }
  }
  if (local) atomicAdd(undecided, local);
}

// Exact sequential finish for whatever the reservation rounds left undecided
// (every earlier-ranked candidate is already final, so the greedy rule can be
// applied in rank order directly).
__global__ void k_select_tail(u32 M, const u32* from, const u32* to, u8* status, u32* role,
                              u32 round) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (u32 r = 0; r < M; ++r) {
    if (status[r] != ST_UNDECIDED) continue;
    u32 A = from[r], B = to[r];
    u32 ba = role_bits(role[A], round), bb = role_bits(role[B], round);
    if ((ba & ROLE_ACC) || (bb & ROLE_EMIT)) {
      status[r] = ST_REJECTED;
      continue;
    }
    status[r] = ST_ACCEPTED;
    role[A] = (round << 2) | (role_bits(role[A], round) | ROLE_EMIT);
    role[B] = (round << 2) | (role_bits(role[B], round) | ROLE_ACC);
  }
}

__global__ void k_cand_flags(const double* gain, u32 na, u8* flag) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < na; i += (u64)gridDim.x * blockDim.x)
    flag[i] = gain[i] > 0.0 ? 1 : 0;
}

__global__ void k_gain_keys(const u32* cidx, u32 M, const double* gain, u64* keys, u32* vals) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < M; i += (u64)gridDim.x * blockDim.x) {
    keys[i] = ~double_key(gain[cidx[i]]);  // descending gain
    vals[i] = cidx[i];
  }
}

__global__ void k_gather_sel(const u32* order, u32 M, const u32* act, const u32* cand_to,
                             const u32* f, u32* sel_node, u32* sel_from, u32* sel_to) {
  for (u64 r = blockIdx.x * (u64)blockDim.x + threadIdx.x; r < M; r += (u64)gridDim.x * blockDim.x) {
    u32 i = order[r];
    u32 v = act[i];
    sel_node[r] = v;
    sel_from[r] = f[v];
    sel_to[r] = cand_to[i];
  }
}

// Apply accepted moves (throughput.rs:182-187).  d(C) changes are exact in
// any order for integral weights; otherwise k_apply_ordered replays them in
// selected order per community.
__global__ void k_apply_moves(u32 M, const u8* status, const u32* sel_node, const u32* sel_from,
                              const u32* sel_to, u32* f, const double* kdeg, double* d,
                              bool atomic_d, u8* changed, u8* affected, bool mark_moved,
                              u32* accepted) {
  u32 local = 0;
  for (u64 r = blockIdx.x * (u64)blockDim.x + threadIdx.x; r < M; r += (u64)gridDim.x * blockDim.x) {
    if (status[r] != ST_ACCEPTED) continue;
    u32 v = sel_node[r];
    f[v] = sel_to[r];
    changed[v] = 1;
    if (mark_moved) affected[v] = 1;
    if (atomic_d) {
      double kv = kdeg[v];
      atomicAdd(&d[sel_from[r]], -kv);
      atomicAdd(&d[sel_to[r]], kv);
    }
    ++local;
  }
  if (local) atomicAdd(accepted, local);
}

__global__ void k_dops(u32 M, const u8* status, const u32* sel_from, const u32* sel_to,
                       u32* okey, u32* oval) {
  for (u64 r = blockIdx.x * (u64)blockDim.x + threadIdx.x; r < M; r += (u64)gridDim.x * blockDim.x) {
    bool acc = status[r] == ST_ACCEPTED;
    okey[2 * r] = acc ? sel_from[r] : NONE32;
    okey[2 * r + 1] = acc ? sel_to[r] : NONE32;
    oval[2 * r] = (u32)(2 * r);
    oval[2 * r + 1] = (u32)(2 * r + 1);
  }
}

// d[c] - k1 + k2 ... in selected order (a - b is a + (-b) exactly).
// The number of segments is read on the device: the exclusive scan of the
// segment heads plus the last head.
__global__ void k_apply_ordered(const u32* seg_last, const u32* head_last, const u32* ukeys,
                                const u32* ustart, u32 total, const u32* ops,
                                const u32* sel_node, const double* kdeg, double* d) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  const u32 nu = *seg_last + *head_last;
  for (u64 j = warp; j < nu; j += nwarps) {
    u32 c = ukeys[j];
    if (c == NONE32) continue;
    u32 a = ustart[j], b = (j + 1 < nu) ? ustart[j + 1] : total;
    double x = warp_ordered_sum(a, b, d[c],
                                [&](u64 t) {
                                  u32 op = ops[t];
                                  double kv = kdeg[sel_node[op >> 1]];
                                  return (op & 1) ? kv : -kv;
                                },
                                [](u64) { return true; });
    if (lane == 0) d[c] = x;
  }
}

// Next frontier and K marks (throughput.rs:189-199), on f after all moves.
// Rows longer than MARK_LONG entries (moved hubs) are cut into segments of
// MARK_LONG entries, listed as (rank, segment) pairs for k_mark_next_long, so
// that no warp walks a row of millions of entries alone while the others idle.
constexpr u64 MARK_LONG = 4096;

// One row's marks over entries [p_lo, p_hi): four entries per lane in
// flight, their neighbours, then their labels.  Returns whether a neighbour
// shares v's sub-community.
__device__ __forceinline__ bool mark_entries(u64 p_lo, u64 p_hi, u32 lane, u32 to, u32 sv,
                                             const u32* col, const u32* f, const u32* s, u8* next,
                                             u8* affected) {
  bool any_same = false;
  for (u64 p0 = p_lo + lane; p0 < p_hi; p0 += 128) {
    u32 nb[4], fn[4], sn[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) nb[j] = p0 + 32 * j < p_hi ? col[p0 + 32 * j] : NONE32;
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (nb[j] != NONE32) {
        fn[j] = f[nb[j]];
        sn[j] = s[nb[j]];
      }
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (nb[j] != NONE32) {
        if (fn[j] != to) next[nb[j]] = 1;
        if (sn[j] == sv) {
          affected[nb[j]] = 1;
          any_same = true;
        }
      }
  }
  return any_same;
}

__global__ void k_mark_next(u32 M, const u8* status, const u32* sel_node, const u32* sel_to,
                            const u64* off, const u32* col, const u32* f, const u32* s, u8* next,
                            u8* affected, unsigned long long* long_list, u32* long_count) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 r = warp; r < M; r += nwarps) {
    if (status[r] != ST_ACCEPTED) continue;
    u32 v = sel_node[r], to = sel_to[r];
    const u64 deg = off[v + 1] - off[v];
    if (deg > MARK_LONG) {
      const u32 nseg = (u32)((deg + MARK_LONG - 1) / MARK_LONG);
      u32 at = 0;
      if (lane == 0) at = atomicAdd(long_count, nseg);
      at = __shfl_sync(0xffffffffu, at, 0);
      for (u32 x = lane; x < nseg; x += 32)
        long_list[at + x] = ((unsigned long long)r << 32) | x;
      continue;
    }
    const bool any_same = mark_entries(off[v], off[v + 1], lane, to, s[v], col, f, s, next,
                                       affected);
    if (__any_sync(0xffffffffu, any_same) && lane == 0) affected[v] = 1;
  }
}

// The segments of long rows k_mark_next listed: a warp per segment, the same
// marks (every segment that meets v's sub-community marks v itself).
__global__ void k_mark_next_long(const unsigned long long* long_list, const u32* long_count,
                                 const u32* sel_node, const u32* sel_to, const u64* off,
                                 const u32* col, const u32* f, const u32* s, u8* next,
                                 u8* affected) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  const u32 cnt = *long_count;
  for (u64 t = warp; t < cnt; t += nwarps) {
    const unsigned long long item = long_list[t];
    const u32 r = (u32)(item >> 32), seg = (u32)item;
    const u32 v = sel_node[r], to = sel_to[r];
    const u64 o0 = off[v], o1 = off[v + 1];
    const u64 lo = o0 + (u64)seg * MARK_LONG;
    const u64 hi = lo + MARK_LONG < o1 ? lo + MARK_LONG : o1;
    const bool any_same = mark_entries(lo, hi, lane, to, s[v], col, f, s, next, affected);
    if (__any_sync(0xffffffffu, any_same) && lane == 0) affected[v] = 1;
  }
}

void ensure_comm_arrays(Engine& E, size_t ncap) {
  Scratch& S = E.sc;
  size_t old_res = S.res.cap, old_role = S.role.cap;
  S.d.ensure(E.mem, ncap);
  S.res.ensure(E.mem, ncap);
  S.role.ensure(E.mem, ncap);
  if (S.res.cap != old_res) HL_CUDA(cudaMemsetAsync(S.res.p, 0, S.res.cap * sizeof(u64), E.stream));
  if (S.role.cap != old_role) HL_CUDA(cudaMemsetAsync(S.role.p, 0, S.role.cap * sizeof(u32), E.stream));
}

// Decides every sorted candidate in S.sel_from / S.sel_to (rank order):
// S.status[r] = accepted / rejected exactly as the sequential greedy would.
void select_decoupled_dev(Engine& E, u32 M) {
  Scratch& S = E.sc;
  cudaStream_t st = E.stream;
  u32* cnt = S.cnt.p;
  cudaEvent_t ev = E.kt_begin();
  HL_CUDA(cudaMemsetAsync(S.status.p, ST_UNDECIDED, M, st));
  u32 round = ++E.sel_round;
  if (round >= (1u << 29)) E.sel_round = round = 1;
  u32 iters = 0;
  while (true) {
    for (int rep = 0; rep < 4; ++rep) {
      u64 e = ++E.epoch;
      HL_CUDA(cudaMemsetAsync(cnt + 6, 0, sizeof(u32), st));
      ++E.nlaunch, k_reserve<<<grid_for(M), 256, 0, st>>>(M, S.sel_from.p, S.sel_to.p, S.status.p, S.nmask.p,
                                             S.role.p, (unsigned long long*)S.res.p, round, e);
      ++E.nlaunch, k_decide<<<grid_for(M), 256, 0, st>>>(M, S.sel_from.p, S.sel_to.p, S.status.p, S.nmask.p,
                                            S.role.p, (const unsigned long long*)S.res.p, round, e,
                                            cnt + 6);
      HL_LAUNCH_CHECK();
      ++iters;
    }
    u32 left = E.read_u32(cnt + 6);
    if (!left) break;
    if (iters >= 64) {
      ++E.nlaunch, k_select_tail<<<1, 32, 0, st>>>(M, S.sel_from.p, S.sel_to.p, S.status.p, S.role.p, round);
      HL_LAUNCH_CHECK();
      break;
    }
  }
  E.stats_sel_iters += iters;
  E.kt_end(KT_SELECT, ev);
  E.kagg[KT_SELECT].bytes += (u64)M * 9 * iters;  // from/to/status/nmask per iteration
}

MoveOut inc_movement(Engine& E, Level& L, const DevEdges& delta, bool all_active,
                     bool mark_moved) {
  MoveOut out;
  Scratch& S = E.sc;
  cudaStream_t st = E.stream;
  const u32 n = L.g.n;
  // flag arrays padded to whole 32-bit words (small.cu marks them by word)
  const size_t nflag = (((size_t)n + 3) & ~(size_t)3) ? (((size_t)n + 3) & ~(size_t)3) : 4;
  S.active.ensure(E.mem, nflag);
  S.next.ensure(E.mem, nflag);
  S.changed.ensure(E.mem, n ? n : 1);
  S.affected.ensure(E.mem, n ? n : 1);
  HL_CUDA(cudaMemsetAsync(S.active.p, all_active ? 1 : 0, n ? n : 1, st));
  HL_CUDA(cudaMemsetAsync(S.changed.p, 0, n ? n : 1, st));
  HL_CUDA(cudaMemsetAsync(S.affected.p, 0, n ? n : 1, st));
  if (!n) return out;
  if (delta.k)
    ++E.nlaunch, k_seed<<<grid_for(delta.k), 256, 0, st>>>(delta.u, delta.v, delta.w, delta.k, L.f.p,
                                               L.s_cur.p, S.active.p, S.affected.p);
  HL_LAUNCH_CHECK();
  if (E.k_flags_set) {  // M8: K marks handed up from the level below
    ++E.nlaunch, k_or_flags<<<grid_for(n), 256, 0, st>>>(S.kflag.p, n, S.affected.p);
    HL_LAUNCH_CHECK();
    E.k_flags_set = false;
  }
  // Community ids must stay below n so that n + v is a fresh empty community.
  compact_labels_if_needed(E, L.f.p, n, n);
  const size_t ncap = 2 * (size_t)n + 2;
  ensure_comm_arrays(E, ncap);
  recompute_comm_degrees(E, L, L.f.p, (u32)ncap, S.d.p);
  if (E.cfg.mode == HL_MODE_DETERMINISTIC) {
    // sequential Gauss–Seidel (hit_leiden.rs:1103-1191): one iteration
    inc_movement_det(E, L, S.d.p, ncap, mark_moved, &out.moves, &out.traversed);
    out.iterations = 1;
    E.kagg[KT_MOVE_EVAL].bytes += 16ull * out.traversed;
    return out;
  }

  S.act.ensure(E.mem, n);
  S.cand_to.ensure(E.mem, n);
  S.cand_gain.ensure(E.mem, n);
  S.cand_idx.ensure(E.mem, n);
  S.status.ensure(E.mem, n);
  S.nmask.ensure(E.mem, n);
  S.sel_node.ensure(E.mem, n);
  S.sel_from.ensure(E.mem, n);
  S.sel_to.ensure(E.mem, n);
  S.order.ensure(E.mem, n);
  S.order2.ensure(E.mem, n);
  S.gkey.ensure(E.mem, n);
  S.gkey2.ensure(E.mem, n);
  S.cnt.ensure(E.mem, 16);
  S.red64.ensure(E.mem, 8);
  HL_CUDA(cudaMemsetAsync(S.red64.p, 0, 8 * sizeof(u64), st));
  u64 sum_nv = 0;
  u32* cnt = S.cnt.p;

  const u32 max_rounds = E.cfg.max_rounds ? E.cfg.max_rounds : 20;
  u32 it = 0;
  S.acc_cnt.ensure(E.mem, 1);
  HL_CUDA(cudaMemsetAsync(S.acc_cnt.p, 0, sizeof(u32), st));  // accepted moves, all rounds
  // Small frontiers run whole rounds in one block (small.cu); the host
  // rounds below take over while the frontier is large or a hub is active.
  u64 sm_moves = 0, sm_cands = 0, sm_trav = 0, sm_nv = 0;
  bool small_on = !(E.cfg.flags & HL_FLAG_NO_SMALL_ROUNDS);
  u32 last_na = 0;
  while (it < max_rounds) {
    if (small_on && last_na <= 16384) {
      bool big = false;
      if (move_rounds_small(E, L, mark_moved, it, sm_moves, sm_cands, sm_trav, sm_nv, &big))
        break;
      if (big) small_on = false;
      if (it >= max_rounds) break;
    }
    // Active list, ascending (iter_ones order).
    cub_run(E, [&](void* t, size_t& b) {
      return cub::DeviceSelect::Flagged(t, b, cub::CountingInputIterator<u32>(0), S.active.p,
                                        S.act.p, cnt + 4, (int64_t)n, st);
    });
    u32 na = E.read_u32(cnt + 4);
    last_na = na;
    if (!na) break;
    sum_nv += na;
    if (!E.in_bootstrap)
      autotune_bins(E, S.act.p, na, L, L.s_cur.p, S.d.p, S.cand_to.p, S.cand_gain.p);
    run_eval(E, EVAL_MOVE, S.act.p, na, L, L.s_cur.p, S.d.p, nullptr, true, S.cand_to.p,
             S.cand_gain.p, (unsigned long long*)S.red64.p);
    // Candidates with positive gain, still in ascending node order.
    u8* flag = S.status.p;
    ++E.nlaunch, k_cand_flags<<<grid_for(na), 256, 0, st>>>(S.cand_gain.p, na, flag);
    HL_LAUNCH_CHECK();
    cub_run(E, [&](void* t, size_t& b) {
      return cub::DeviceSelect::Flagged(t, b, cub::CountingInputIterator<u32>(0), flag,
                                        S.cand_idx.p, cnt + 5, (int64_t)na, st);
    });
    u32 M = E.read_u32(cnt + 5);
    out.candidates += M;
    ++it;
    if (!M) break;  // no positive candidate: nothing selected, frontier empties
    ++E.nlaunch, k_gain_keys<<<grid_for(M), 256, 0, st>>>(S.cand_idx.p, M, S.cand_gain.p, S.gkey.p, S.order.p);
    HL_LAUNCH_CHECK();
    {
      u64* ki = S.gkey.p;
      u64* ko = S.gkey2.p;
      u32* vi = S.order.p;
      u32* vo = S.order2.p;
      cub_run(E, [&](void* t, size_t& b) {
        return cub::DeviceRadixSort::SortPairs(t, b, ki, ko, vi, vo, (int64_t)M, 0, 64, st);
      });
    }
    ++E.nlaunch, k_gather_sel<<<grid_for(M), 256, 0, st>>>(S.order2.p, M, S.act.p, S.cand_to.p, L.f.p,
                                              S.sel_node.p, S.sel_from.p, S.sel_to.p);
    HL_LAUNCH_CHECK();
    select_decoupled_dev(E, M);
    cudaEvent_t ev_mark = E.kt_begin();
    ++E.nlaunch, k_apply_moves<<<grid_for(M), 256, 0, st>>>(M, S.status.p, S.sel_node.p, S.sel_from.p,
                                               S.sel_to.p, L.f.p, L.k.p, S.d.p, E.integral,
                                               S.changed.p, S.affected.p, mark_moved, S.acc_cnt.p);
    HL_LAUNCH_CHECK();
    if (!E.integral) {
      // Replay d(C) -= k / += k in selected order, per community.
      S.used.ensure(E.mem, 2 * (size_t)M);
      S.rank.ensure(E.mem, 2 * (size_t)M);
      S.cand_node.ensure(E.mem, 2 * (size_t)M);
      S.segid.ensure(E.mem, 2 * (size_t)M);
      S.rowlist.ensure(E.mem, 2 * (size_t)M);
      S.seg_start.ensure(E.mem, 2 * (size_t)M);
      S.idx.ensure(E.mem, 2 * (size_t)M);
      S.idx2.ensure(E.mem, 2 * (size_t)M);
      ++E.nlaunch, k_dops<<<grid_for(M), 256, 0, st>>>(M, S.status.p, S.sel_from.p, S.sel_to.p, S.used.p,
                                          S.idx.p);
      HL_LAUNCH_CHECK();
      u32 M2 = 2 * M;
      u32* ki = S.used.p;
      u32* ko = S.rank.p;
      u32* vi = S.idx.p;
      u32* vo = S.idx2.p;
      cub_run(E, [&](void* t, size_t& b) {
        return cub::DeviceRadixSort::SortPairs(t, b, ki, ko, vi, vo, (int64_t)M2, 0, 32, st);
      });
      ++E.nlaunch, k_heads_u32<<<grid_for(M2), 256, 0, st>>>(ko, M2, S.cand_node.p);
      HL_LAUNCH_CHECK();
      u32* h = S.cand_node.p;
      u32* sid = S.segid.p;
      cub_run(E, [&](void* t, size_t& b) {
        return cub::DeviceScan::ExclusiveSum(t, b, h, sid, (int64_t)M2, st);
      });
      ++E.nlaunch, k_seg_compact<<<grid_for(M2), 256, 0, st>>>(h, sid, ko, M2, S.rowlist.p, S.seg_start.p);
      ++E.nlaunch, k_apply_ordered<<<grid_for((u64)M2 * 32), 256, 0, st>>>(
          sid + M2 - 1, h + M2 - 1, S.rowlist.p, S.seg_start.p, M2, vo, S.sel_node.p, L.k.p, S.d.p);
      HL_LAUNCH_CHECK();
    }
    // No early exit on zero accepted moves (it would cost a read-back every
    // round): such a round marks nothing, so the next frontier is empty and
    // the loop ends on it with the same iteration count.
    HL_CUDA(cudaMemsetAsync(S.next.p, 0, n, st));
    // segments of the long rows: at most M + nnz / MARK_LONG
    S.mark_long.ensure(E.mem, (size_t)M + L.g.nnz / MARK_LONG + 1);
    S.mark_long_cnt.ensure(E.mem, 1);
    HL_CUDA(cudaMemsetAsync(S.mark_long_cnt.p, 0, sizeof(u32), st));
    ++E.nlaunch, k_mark_next<<<grid_for((u64)M * 32), 256, 0, st>>>(M, S.status.p, S.sel_node.p, S.sel_to.p,
                                                        L.g.off.p, L.g.col.p, L.f.p, L.s_cur.p,
                                                        S.next.p, S.affected.p, S.mark_long.p,
                                                        S.mark_long_cnt.p);
    ++E.nlaunch, k_mark_next_long<<<148 * 8, 256, 0, st>>>(S.mark_long.p, S.mark_long_cnt.p,
                                                           S.sel_node.p,
                                                           S.sel_to.p, L.g.off.p, L.g.col.p,
                                                           L.f.p, L.s_cur.p, S.next.p,
                                                           S.affected.p);
    HL_LAUNCH_CHECK();
    E.kt_end(KT_MARK_NEXT, ev_mark);
    S.active.swap(S.next);
  }
  out.iterations = it;
  // The evaluation counters and the accepted moves stay on the device until
  // the call ends (Scratch::bacc; the algorithmic bytes are counted there).
  stats_acc_u64(E, reinterpret_cast<const unsigned long long*>(S.red64.p), 8, 0);
  stats_acc_u32(E, S.acc_cnt.p, 8);
  E.sum_nv_batch += sum_nv;
  out.moves += sm_moves;
  out.candidates += sm_cands;
  out.traversed += sm_trav;
  return out;
}

}  // namespace hl
