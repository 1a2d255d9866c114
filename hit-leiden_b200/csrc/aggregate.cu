// aggregate.cu — inc-aggregation (hit_leiden.rs:1639-1731), the bootstrap
// aggregation, and the level maps (def-update, hit_leiden.rs:1733-1793).
//
// ΔH records are emitted at fixed positions that follow the reference's push
// order (the lifted ΔG first, then per refined vertex in ascending order its
// adjacency in CSR order, then its self-loop pair).  A stable radix sort on the
// (min, max) key followed by an in-order segmented sum reproduces Compress()'s
// per-key rounding exactly; entries with |w| <= 1e-9 are dropped and the
// result comes out in ascending key order.
#include "hl_engine.cuh"

namespace hl {

static inline u32 grid_for(u64 n, u32 block = 256) {
  u64 g = (n + block - 1) / block;
  if (g > 148u * 64u) g = 148u * 64u;
  return g ? (u32)g : 1u;
}

__device__ __forceinline__ bool agg_vertex(u32 v, const u8* refined, const u32* s_pre,
                                           const u32* s_cur, bool changed_only) {
  return refined[v] && (!changed_only || s_cur[v] != s_pre[v]);
}

__device__ __forceinline__ bool agg_emit(u32 v, u32 nb, const u8* refined, const u32* s_pre,
                                         const u32* s_cur, bool changed_only) {
  if (s_cur[nb] == s_pre[nb] || v < nb) return true;
  return changed_only && !refined[nb];
}

__device__ __forceinline__ u64 pair_key(u32 a, u32 b) {
  return a <= b ? (((u64)a << 32) | b) : (((u64)b << 32) | a);
}

__global__ void k_agg_lift(const u32* u, const u32* v, const double* w, u64 k, const u32* s_pre,
                           u64* keys, double* vals, u32* seq) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < k; i += (u64)gridDim.x * blockDim.x) {
    keys[i] = pair_key(s_pre[u[i]], s_pre[v[i]]);
    vals[i] = w ? w[i] : 1.0;
    seq[i] = (u32)i;
  }
}

// Warp per refined vertex: its adjacency is scanned 32 entries at a time in
// CSR order; each emitting entry writes its (-w, +w) pair at the position
// given by the ballot prefix, so the records keep the reference's push order.
// With `pos == nullptr` only the per-vertex record count is produced.
__global__ void k_agg_rows(u32 n, const u64* off, const u32* col, const double* w,
                           const u8* refined, const u32* s_pre, const u32* s_cur,
                           bool changed_only, bool edge_weight_loops, u64* cnt, const u64* pos,
                           u64 base, u64* keys, double* vals, u32* seq) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 v = warp; v < n; v += nwarps) {
    if (!agg_vertex((u32)v, refined, s_pre, s_cur, changed_only)) {
      if (!pos && lane == 0) cnt[v] = 0;
      continue;
    }
    const u64 o0 = off[v], o1 = off[v + 1];
    const u32 sp = s_pre[v], sc = s_cur[v];
    u64 o = pos ? base + pos[v] : 0;
    u64 c = 0;
    // Four chunks per step: their neighbours, then their labels, are loaded
    // before any is decided, so a long row keeps several gathers in flight;
    // the chunks' records are then placed in CSR order.
    for (u64 b0 = o0; b0 < o1; b0 += 128) {
      u32 nb[4], np_[4], nc[4];
      u8 rf[4];
      double x[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const u64 p = b0 + 32 * j + lane;
        nb[j] = p < o1 ? col[p] : NONE32;
        x[j] = p < o1 ? w[p] : 0.0;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (nb[j] != NONE32) {
          np_[j] = s_pre[nb[j]];
          nc[j] = s_cur[nb[j]];
          rf[j] = refined[nb[j]];
        }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        // agg_emit on the gathered labels
        const bool emit = nb[j] != NONE32 && nb[j] != (u32)v &&
                          (nc[j] == np_[j] || (u32)v < nb[j] || (changed_only && !rf[j]));
        const u32 m = __ballot_sync(0xffffffffu, emit);
        if (pos && emit) {
          const u64 at = o + 2ull * __popc(m & ((1u << lane) - 1u));
          keys[at] = pair_key(sp, np_[j]);
          vals[at] = -x[j];
          seq[at] = (u32)at;
          keys[at + 1] = pair_key(sc, nc[j]);
          vals[at + 1] = x[j];
          seq[at + 1] = (u32)(at + 1);
        }
        o += 2ull * __popc(m);
        c += 2ull * __popc(m);
      }
    }
    // The self-loop's entries (stored twice) sit together at the lower bound
    // of v in the sorted row; their sum in CSR order is the row-order sum of
    // the entries whose neighbour is v.
    double slw = 0.0;
    for (u64 p = lower_bound_u32(col, o0, o1, (u32)v); p < o1 && col[p] == (u32)v; ++p)
      slw = __dadd_rn(slw, w[p]);
    if (edge_weight_loops) slw = slw / 2.0;
    bool loop = fabs(slw) > 1e-12;
    if (lane == 0) {
      if (!pos) {
        cnt[v] = c + (loop ? 2 : 0);
      } else if (loop) {
        keys[o] = pair_key(sp, sp);
        vals[o] = -slw;
        seq[o] = (u32)o;
        keys[o + 1] = pair_key(sc, sc);
        vals[o + 1] = slw;
        seq[o + 1] = (u32)(o + 1);
      }
    }
  }
}

__global__ void k_heads64(const u64* sk, u64 n, u32* head) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    head[i] = (i == 0 || sk[i] != sk[i - 1]) ? 1u : 0u;
}

__global__ void k_seg_start64(const u32* head, const u32* segid, u64 n, u32* start) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    if (head[i]) start[segid[i]] = (u32)i;
}

// One compressed record: the key of segment j (starting at a), its sum x.
__device__ __forceinline__ void compress_out(u64 j, u64 a, double x, const u64* sk,
                                             double threshold, u32* ou, u32* ov, double* ow,
                                             u8* keepf) {
  if ((threadIdx.x & 31) == 0) {
    u64 key = sk[a];
    ou[j] = (u32)(key >> 32);
    ov[j] = (u32)key;
    ow[j] = x;
    keepf[j] = fabs(x) > threshold ? 1 : 0;
  }
}

// In-order segmented sum over the records' weights gathered into sorted
// order (sw); keep |w| > threshold.  Segments of RUN_FOLD_MIN or more terms
// are listed for k_compress_runs.
__global__ void k_compress(u32 U, const u32* start, u64 total, const u64* sk, const double* sw,
                           double threshold, u32* ou, u32* ov, double* ow, u8* keepf, u32* longl,
                           u32* longn) {
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 j = warp; j < U; j += nwarps) {
    u64 a = start[j], b = (j + 1 < U) ? start[j + 1] : total;
    if (b - a >= RUN_FOLD_MIN) {
      fold_defer(longl, longn, (u32)j);
      continue;
    }
    double x = 0.0;
    if (b - a == 1) {
      x = sw[a];
    } else {
      x = warp_ordered_sum(a, b, 0.0, [&](u64 t) { return sw[t]; }, [](u64) { return true; });
    }
    compress_out(j, a, x, sk, threshold, ou, ov, ow, keepf);
  }
}

// The long segments listed by k_compress, folded in runs (the same bits).
__global__ void k_compress_runs(const u32* longl, const u32* longn, u32 U, const u32* start,
                                u64 total, const u64* sk, const double* sw, double threshold,
                                u32* ou, u32* ov, double* ow, u8* keepf) {
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  const u32 nl = *longn;
  for (u64 i = warp; i < nl; i += nwarps) {
    const u32 j = longl[i];
    u64 a = start[j], b = (j + 1 < U) ? start[j + 1] : total;
    double x = warp_fold_runs(a, b, 0.0, sw);
    compress_out(j, a, x, sk, threshold, ou, ov, ow, keepf);
  }
}

// out[t] = src[idx[t]]: the weights gathered into the records' sorted order.
__global__ void k_gather_weights(const u32* idx, const double* src, u64 n, double* out) {
  for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < n; t += (u64)gridDim.x * blockDim.x)
    out[t] = src[idx[t]];
}

__global__ void k_set_spre(u32 n, const u8* refined, const u32* s_cur, u32* s_pre) {
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x)
    if (refined[v]) s_pre[v] = s_cur[v];
}

// Sort (key, seq) records, sum each key in push order, drop |w| <= threshold.
// Output edges land in sc.eu2 / ev2 / ew2 in ascending key order.
// Keys are pair_key(a, b) of ids below id_bound.
static u64 compress_records(Engine& E, u64 R, double threshold, u32 id_bound) {
  Scratch& S = E.sc;
  cudaStream_t st = E.stream;
  if (!R) return 0;
  u64* ki = S.keys.p;
  u64* ko = S.keys2.p;
  u32* vi = S.idx.p;
  u32* vo = S.idx2.p;
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceRadixSort::SortPairs(t, b, ki, ko, vi, vo, (int64_t)R, 0,
                                           32 + bits_for(id_bound ? id_bound - 1 : 0), st);
  });
  S.rowlist.ensure(E.mem, R);
  S.segid.ensure(E.mem, R);
  S.seg_start.ensure(E.mem, R);
  ++E.nlaunch, k_heads64<<<grid_for(R), 256, 0, st>>>(ko, R, S.rowlist.p);
  HL_LAUNCH_CHECK();
  u32* h = S.rowlist.p;
  u32* sid = S.segid.p;
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceScan::ExclusiveSum(t, b, h, sid, (int64_t)R, st);
  });
  u32 uh[2];
  E.read_u32s({sid + R - 1, h + R - 1}, uh);
  const u32 U = uh[0] + uh[1];
  ++E.nlaunch, k_seg_start64<<<grid_for(R), 256, 0, st>>>(h, sid, R, S.seg_start.p);
  S.eu.ensure(E.mem, U);
  S.ev.ensure(E.mem, U);
  S.ew.ensure(E.mem, U);
  S.op.ensure(E.mem, U);
  S.fvals.ensure(E.mem, R);
  ++E.nlaunch, k_gather_weights<<<grid_for(R), 256, 0, st>>>(vo, S.neww.p, R, S.fvals.p);
  FoldList fl = fold_list(E, R, U);
  ++E.nlaunch, k_compress<<<grid_for((u64)U * 32), 256, 0, st>>>(
      U, S.seg_start.p, R, ko, S.fvals.p, threshold, S.eu.p, S.ev.p, S.ew.p, S.op.p, fl.seg,
      fl.cnt);
  ++E.nlaunch, k_compress_runs<<<FOLD_BLOCKS, 256, 0, st>>>(
      fl.seg, fl.cnt, U, S.seg_start.p, R, ko, S.fvals.p, threshold, S.eu.p, S.ev.p, S.ew.p,
      S.op.p);
  HL_LAUNCH_CHECK();
  S.eu2.ensure(E.mem, U);
  S.ev2.ensure(E.mem, U);
  S.ew2.ensure(E.mem, U);
  u32* cnt = S.cnt.p + 10;
  u32* a = S.eu.p;
  u32* a2 = S.eu2.p;
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceSelect::Flagged(t, b, a, S.op.p, a2, cnt, (int64_t)U, st);
  });
  u32* c = S.ev.p;
  u32* c2 = S.ev2.p;
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceSelect::Flagged(t, b, c, S.op.p, c2, cnt, (int64_t)U, st);
  });
  double* d = S.ew.p;
  double* d2 = S.ew2.p;
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceSelect::Flagged(t, b, d, S.op.p, d2, cnt, (int64_t)U, st);
  });
  return E.read_u32(cnt);
}

u64 inc_aggregation(Engine& E, Level& L, const DevEdges& delta, u32* next_n, bool changed_only,
                    bool edge_weight_loops) {
  Scratch& S = E.sc;
  cudaStream_t st = E.stream;
  const u32 n = L.g.n;
  cudaEvent_t kev = E.kt_begin();
  // next node count from the maps before s_pre is updated (:1716-1722)
  S.cnt.ensure(E.mem, 16);
  {
    u32* o = S.cnt.p + 12;
    u32* sp = L.s_pre.p;
    u32* sc = L.s_cur.p;
    u32 m1 = 0, m2 = 0;
    if (n) {
      cub_run(E, [&](void* t, size_t& b) {
        return cub::DeviceReduce::Max(t, b, sp, o, (int64_t)n, st);
      });
      cub_run(E, [&](void* t, size_t& b) {
        return cub::DeviceReduce::Max(t, b, sc, o + 1, (int64_t)n, st);
      });
      u32 mm[2];
      E.read_u32s({o, o + 1}, mm);
      m1 = mm[0];
      m2 = mm[1];
    }
    *next_n = (m1 > m2 ? m1 : m2) + 1;
  }
  S.newoff.ensure(E.mem, (size_t)n + 1);
  S.gkey2.ensure(E.mem, (size_t)n + 1);
  ++E.nlaunch, k_agg_rows<<<grid_for((u64)n * 32), 256, 0, st>>>(
      n, L.g.off.p, L.g.col.p, L.g.w.p, S.refined.p, L.s_pre.p, L.s_cur.p, changed_only,
      edge_weight_loops, S.newoff.p, nullptr, 0, nullptr, nullptr, nullptr);
  HL_CUDA(cudaMemsetAsync(S.newoff.p + n, 0, sizeof(u64), st));
  HL_LAUNCH_CHECK();
  u64* a = S.newoff.p;
  u64* pos = S.gkey2.p;
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceScan::ExclusiveSum(t, b, a, pos, (int64_t)n + 1, st);
  });
  u64 R2 = E.read_u64(pos + n);
  u64 R = delta.k + R2;
  if (R) {
    S.keys.ensure(E.mem, R);
    S.keys2.ensure(E.mem, R);
    S.idx.ensure(E.mem, R);
    S.idx2.ensure(E.mem, R);
    S.neww.ensure(E.mem, R);
    if (delta.k)
      ++E.nlaunch, k_agg_lift<<<grid_for(delta.k), 256, 0, st>>>(delta.u, delta.v, delta.w, delta.k, L.s_pre.p,
                                                    S.keys.p, S.neww.p, S.idx.p);
    ++E.nlaunch, k_agg_rows<<<grid_for((u64)n * 32), 256, 0, st>>>(
        n, L.g.off.p, L.g.col.p, L.g.w.p, S.refined.p, L.s_pre.p, L.s_cur.p, changed_only,
        edge_weight_loops, nullptr, pos, delta.k, S.keys.p, S.neww.p, S.idx.p);
    HL_LAUNCH_CHECK();
  }
  u64 out = compress_records(E, R, 1e-9, *next_n);
  ++E.nlaunch, k_set_spre<<<grid_for(n), 256, 0, st>>>(n, S.refined.p, L.s_cur.p, L.s_pre.p);
  HL_LAUNCH_CHECK();
  E.kt_end(KT_AGGREGATE, kev);
  // ΔG lifted (u, v, w + two s_pre reads), refined rows scanned (maps, row
  // entries), ΔH records written and read once, compressed output written.
  E.kagg[KT_AGGREGATE].bytes += 32ull * delta.k + 13ull * n + 10ull * (L.g.nnz ? R2 / 2 : 0) * 2 +
                                 32ull * R + 16ull * out;
  return out;
}

// Bootstrap aggregation of G^p by s: every undirected edge once (a self-loop
// counted once), summed per (s(u), s(v)) in (u ascending, CSR) order.
__global__ void k_full_count(u32 n, const u64* off, const u32* col, u64* cnt) {
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x) {
    u64 c = 0;
    for (u64 p = off[v]; p < off[v + 1]; ++p) {
      u32 nb = col[p];
      if (nb < v) continue;
      if (nb == v && p + 1 < off[v + 1] && col[p + 1] == (u32)v) continue;
      ++c;
    }
    cnt[v] = c;
  }
}

__global__ void k_full_emit(u32 n, const u64* off, const u32* col, const double* w, const u32* s,
                            const u64* pos, u64* keys, double* vals, u32* seq) {
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x) {
    u64 o = pos[v];
    for (u64 p = off[v]; p < off[v + 1]; ++p) {
      u32 nb = col[p];
      if (nb < v) continue;
      if (nb == v && p + 1 < off[v + 1] && col[p + 1] == (u32)v) continue;
      keys[o] = pair_key(s[v], s[nb]);
      vals[o] = w[p];
      seq[o] = (u32)o;
      ++o;
    }
  }
}

u64 aggregate_full(Engine& E, Level& L, const u32* s, u32*, u32*, double*) {
  Scratch& S = E.sc;
  cudaStream_t st = E.stream;
  const u32 n = L.g.n;
  S.newoff.ensure(E.mem, (size_t)n + 1);
  S.gkey2.ensure(E.mem, (size_t)n + 1);
  ++E.nlaunch, k_full_count<<<grid_for(n), 256, 0, st>>>(n, L.g.off.p, L.g.col.p, S.newoff.p);
  HL_CUDA(cudaMemsetAsync(S.newoff.p + n, 0, sizeof(u64), st));
  HL_LAUNCH_CHECK();
  u64* a = S.newoff.p;
  u64* pos = S.gkey2.p;
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceScan::ExclusiveSum(t, b, a, pos, (int64_t)n + 1, st);
  });
  u64 R = E.read_u64(pos + n);
  if (!R) return 0;
  S.keys.ensure(E.mem, R);
  S.keys2.ensure(E.mem, R);
  S.idx.ensure(E.mem, R);
  S.idx2.ensure(E.mem, R);
  S.neww.ensure(E.mem, R);
  ++E.nlaunch, k_full_emit<<<grid_for(n), 256, 0, st>>>(n, L.g.off.p, L.g.col.p, L.g.w.p, s, pos, S.keys.p,
                                           S.neww.p, S.idx.p);
  HL_LAUNCH_CHECK();
  return compress_records(E, R, -1.0, n);
}

// f^{p+1}(s^p(v)) := f^p(v); with several members the largest v writes last,
// exactly like the sequential loop.
__global__ void k_last_member(u32 n, const u32* s, u32* last) {
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x)
    atomicMax(&last[s[v]], (u32)v + 1);
}
__global__ void k_project(u32 nh, const u32* last, const u32* flo, u32* fhi, u8* changed) {
  for (u64 x = blockIdx.x * (u64)blockDim.x + threadIdx.x; x < nh; x += (u64)gridDim.x * blockDim.x) {
    u32 l = last[x];
    if (!l) continue;
    const u32 nf = flo[l - 1];
    if (fhi[x] != nf) {
      fhi[x] = nf;
      if (changed) changed[x] = 1;  // M8: its sub-community is split again above
    }
  }
}

void project_up(Engine& E, Level& lo, Level& hi, u8* changed_flags) {
  Scratch& S = E.sc;
  u32 nh = hi.g.n;
  S.minmem.ensure(E.mem, (size_t)nh + 1);
  HL_CUDA(cudaMemsetAsync(S.minmem.p, 0, sizeof(u32) * ((size_t)nh + 1), E.stream));
  ++E.nlaunch, k_last_member<<<grid_for(lo.g.n), 256, 0, E.stream>>>(lo.g.n, lo.s_cur.p, S.minmem.p);
  ++E.nlaunch, k_project<<<grid_for(nh), 256, 0, E.stream>>>(nh, S.minmem.p, lo.f.p, hi.f.p,
                                                              changed_flags);
  HL_LAUNCH_CHECK();
}

__global__ void k_top_down(u32 n, const u32* s, const u32* fhi, const u32* ghi, u32* flo,
                           u32* glo) {
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x) {
    u32 x = s[v];
    flo[v] = fhi[x];
    glo[v] = ghi[x];
  }
}

void top_down(Engine& E) {
  int P = (int)E.levels.size();
  Level& top = E.levels[P - 1];
  ++E.nlaunch, k_iota<<<grid_for(top.g.n), 256, 0, E.stream>>>(top.gm.p, top.g.n);
  for (int p = P - 2; p >= 0; --p) {
    Level& lo = E.levels[p];
    Level& hi = E.levels[p + 1];
    ++E.nlaunch, k_top_down<<<grid_for(lo.g.n), 256, 0, E.stream>>>(lo.g.n, lo.s_cur.p, hi.f.p, hi.gm.p, lo.f.p,
                                                        lo.gm.p);
  }
  HL_LAUNCH_CHECK();
}

__global__ void k_inherit(const u32* xs, const u32* os, u32 m, u32* s_pre, u32* s_cur, u32* gm) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < m; i += (u64)gridDim.x * blockDim.x) {
    u32 x = xs[i], o = os[i];
    s_pre[x] = s_pre[o];
    s_cur[x] = s_cur[o];
    gm[x] = gm[o];
  }
}

void inherit_new_nodes(Engine& E, Level& hi, const std::vector<std::pair<u32, u32>>& ids) {
  if (ids.empty()) return;
  u32 m = (u32)ids.size();
  std::vector<u32> xs(m), os(m);
  for (u32 i = 0; i < m; ++i) {
    xs[i] = ids[i].first;
    os[i] = ids[i].second;
  }
  Scratch& S = E.sc;
  S.upd_node.ensure(E.mem, m);
  S.upd_to.ensure(E.mem, m);
  HL_CUDA(cudaMemcpyAsync(S.upd_node.p, xs.data(), sizeof(u32) * m, cudaMemcpyHostToDevice, E.stream));
  HL_CUDA(cudaMemcpyAsync(S.upd_to.p, os.data(), sizeof(u32) * m, cudaMemcpyHostToDevice, E.stream));
  ++E.nlaunch, k_inherit<<<grid_for(m), 256, 0, E.stream>>>(S.upd_node.p, S.upd_to.p, m, hi.s_pre.p, hi.s_cur.p,
                                               hi.gm.p);
  HL_LAUNCH_CHECK();
  E.sync();  // host vectors go out of scope
}

}  // namespace hl
