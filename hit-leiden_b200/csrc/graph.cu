// graph.cu — device CSR maintenance: G ← G ⊕ ΔG (K1), degrees, 2m.
//
// apply_delta restates in_memory.rs:103-137: every ΔG edge is keyed by
// (min, max); a key's new weight is its existing weight followed by the
// batch's deltas in batch order (a stable sort keeps that order); keys whose
// weight ends at <= 1e-12 disappear.  Instead of rebuilding a hash map of all
// m edges, only the changed keys are resolved: weight updates are written in
// place, and inserts/deletes become sorted row-operations that a warp-per-row
// merge folds into a fresh CSR with rows still sorted by neighbour id.
#include "hl_engine.cuh"

namespace hl {

__global__ void k_fill_u8(u8* p, u8 v, u64 n) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    p[i] = v;
}

__global__ void k_iota(u32* p, u32 n) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    p[i] = (u32)i;
}

__global__ void k_fill_u64_range(u64* p, u64 v, u64 lo, u64 hi) {
  for (u64 i = lo + blockIdx.x * (u64)blockDim.x + threadIdx.x; i < hi;
       i += (u64)gridDim.x * blockDim.x)
    p[i] = v;
}

__global__ void k_fill_f64_range(double* p, double v, u64 lo, u64 hi) {
  for (u64 i = lo + blockIdx.x * (u64)blockDim.x + threadIdx.x; i < hi;
       i += (u64)gridDim.x * blockDim.x)
    p[i] = v;
}

__global__ void k_iota_range(u32* p, u64 lo, u64 hi) {
  for (u64 i = lo + blockIdx.x * (u64)blockDim.x + threadIdx.x; i < hi;
       i += (u64)gridDim.x * blockDim.x)
    p[i] = (u32)i;
}

static inline u32 grid_for(u64 n, u32 block = 256) {
  u64 g = (n + block - 1) / block;
  if (g > 148u * 64u) g = 148u * 64u;
  return g ? (u32)g : 1u;
}

void graph_init_empty(Engine& E, Level& L, u32 n) {
  L.g.n = n;
  L.g.nnz = 0;
  L.g.self_loop_entries = 0;
  L.g.off.ensure(E.mem, (size_t)n + 1);
  HL_CUDA(cudaMemsetAsync(L.g.off.p, 0, sizeof(u64) * ((size_t)n + 1), E.stream));
  L.g.col.ensure(E.mem, 1);
  L.g.w.ensure(E.mem, 1);
  L.f.ensure(E.mem, n ? n : 1);
  L.gm.ensure(E.mem, n ? n : 1);
  L.s_pre.ensure(E.mem, n ? n : 1);
  L.s_cur.ensure(E.mem, n ? n : 1);
  L.k.ensure(E.mem, n ? n : 1);
  if (n) {
    ++E.nlaunch, k_iota<<<grid_for(n), 256, 0, E.stream>>>(L.f.p, n);
    ++E.nlaunch, k_iota<<<grid_for(n), 256, 0, E.stream>>>(L.gm.p, n);
    ++E.nlaunch, k_iota<<<grid_for(n), 256, 0, E.stream>>>(L.s_pre.p, n);
    ++E.nlaunch, k_iota<<<grid_for(n), 256, 0, E.stream>>>(L.s_cur.p, n);
    HL_CUDA(cudaMemsetAsync(L.k.p, 0, sizeof(double) * n, E.stream));
  }
  L.tw = 0.0;
  HL_LAUNCH_CHECK();
}

// New nodes start isolated with identity maps (PartitionState::identity).
void graph_grow_nodes(Engine& E, Level& L, u32 n) {
  u32 old = L.g.n;
  if (n <= old) return;
  L.g.off.ensure(E.mem, (size_t)n + 1, true);
  ++E.nlaunch, k_fill_u64_range<<<grid_for(n - old), 256, 0, E.stream>>>(L.g.off.p, L.g.nnz, (u64)old + 1,
                                                             (u64)n + 1);
  L.f.ensure(E.mem, n, true);
  L.gm.ensure(E.mem, n, true);
  L.s_pre.ensure(E.mem, n, true);
  L.s_cur.ensure(E.mem, n, true);
  L.k.ensure(E.mem, n, true);
  ++E.nlaunch, k_iota_range<<<grid_for(n - old), 256, 0, E.stream>>>(L.f.p, old, n);
  ++E.nlaunch, k_iota_range<<<grid_for(n - old), 256, 0, E.stream>>>(L.gm.p, old, n);
  ++E.nlaunch, k_iota_range<<<grid_for(n - old), 256, 0, E.stream>>>(L.s_pre.p, old, n);
  ++E.nlaunch, k_iota_range<<<grid_for(n - old), 256, 0, E.stream>>>(L.s_cur.p, old, n);
  ++E.nlaunch, k_fill_f64_range<<<grid_for(n - old), 256, 0, E.stream>>>(L.k.p, 0.0, old, n);
  L.g.n = n;
  HL_LAUNCH_CHECK();
}

__device__ __forceinline__ u64 lower_bound_u64(const u64* a, u64 lo, u64 hi, u64 x) {
  while (lo < hi) {
    u64 mid = (lo + hi) >> 1;
    if (a[mid] < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

__global__ void k_check_endpoints(const u32* u, const u32* v, u64 k, u32 n, u32* bad) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < k; i += (u64)gridDim.x * blockDim.x)
    if (u[i] >= n || v[i] >= n) atomicAdd(bad, 1u);
}

void check_endpoints(Engine& E, const DevEdges& b, u32 n) {
  if (!b.k) return;
  E.sc.cnt.ensure(E.mem, 16);
  HL_CUDA(cudaMemsetAsync(E.sc.cnt.p, 0, sizeof(u32), E.stream));
  ++E.nlaunch, k_check_endpoints<<<grid_for(b.k), 256, 0, E.stream>>>(b.u, b.v, b.k, n, E.sc.cnt.p);
  HL_LAUNCH_CHECK();
  u32 bad = E.read_u32(E.sc.cnt.p);
  require(bad == 0, "edge endpoint exceeds node_count (" + std::to_string(bad) + " edges)");
}

__global__ void k_integral(const double* w, u64 k, u32* bad) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < k; i += (u64)gridDim.x * blockDim.x) {
    double x = w[i];
    if (!(x == floor(x)) || fabs(x) > 4294967296.0) atomicAdd(bad, 1u);
  }
}

bool edges_integral(Engine& E, const DevEdges& b) {
  if (!b.k || !b.w) return true;
  E.sc.cnt.ensure(E.mem, 16);
  HL_CUDA(cudaMemsetAsync(E.sc.cnt.p + 1, 0, sizeof(u32), E.stream));
  ++E.nlaunch, k_integral<<<grid_for(b.k), 256, 0, E.stream>>>(b.w, b.k, E.sc.cnt.p + 1);
  HL_LAUNCH_CHECK();
  return E.read_u32(E.sc.cnt.p + 1) == 0;
}

__global__ void k_delta_keys(const u32* u, const u32* v, u64 k, u64* keys, u32* idx) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < k; i += (u64)gridDim.x * blockDim.x) {
    u32 a = u[i], b = v[i];
    u32 lo = a < b ? a : b, hi = a < b ? b : a;
    keys[i] = ((u64)lo << 32) | hi;
    idx[i] = (u32)i;
  }
}

__global__ void k_heads(const u64* sk, u64 k, u32* head) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < k; i += (u64)gridDim.x * blockDim.x)
    head[i] = (i == 0 || sk[i] != sk[i - 1]) ? 1u : 0u;
}

__global__ void k_seg_start(const u32* head, const u32* segid, u64 k, u32* seg_start) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < k; i += (u64)gridDim.x * blockDim.x)
    if (head[i]) seg_start[segid[i]] = (u32)i;
}

enum : u8 { OP_NONE = 0, OP_UPD = 1, OP_INS = 2, OP_DEL = 3 };

// One thread per distinct key: existing weight, then the batch's deltas in
// batch order (in_memory.rs:133-137), then the > 1e-12 filter (:110).
__global__ void k_resolve(u32 U, const u32* seg_start, u64 k, const u64* sk, const u32* sidx,
                          const double* bw, const u64* off, const u32* col, double* w,
                          bool keep_loops, u8* op, double* neww, u8* ktouched, u32* nops_del,
                          u32* nops_ins, u32* loop_counts) {
  for (u64 j = blockIdx.x * (u64)blockDim.x + threadIdx.x; j < U; j += (u64)gridDim.x * blockDim.x) {
    u64 t0 = seg_start[j];
    u64 t1 = (j + 1 < U) ? seg_start[j + 1] : k;
    u64 key = sk[t0];
    u32 a = (u32)(key >> 32), b = (u32)key;
    u64 o0 = off[a], o1 = off[a + 1];
    u64 p = lower_bound_u32(col, o0, o1, b);
    bool present = p < o1 && col[p] == b;
    if (a == b && !keep_loops) present = false;
    double x = present ? w[p] : 0.0;
    for (u64 t = t0; t < t1; ++t) x = __dadd_rn(x, bw ? bw[sidx[t]] : 1.0);
    u8 o = OP_NONE;
    u32 nd = 0, ni = 0;
    if (present) {
      if (x > 1e-12) {
        o = OP_UPD;
        w[p] = x;
        if (a == b) {
          w[p + 1] = x;
        } else {
          u64 q = lower_bound_u32(col, off[b], off[b + 1], a);
          w[q] = x;
        }
      } else {
        o = OP_DEL;
        nd = 2;
        if (a == b) atomicAdd(&loop_counts[1], 1u);
      }
    } else if (x > 1e-12) {
      o = OP_INS;
      ni = 2;
      if (a == b) atomicAdd(&loop_counts[0], 1u);
    }
    op[j] = o;
    neww[j] = x;
    nops_del[j] = nd;
    nops_ins[j] = ni;
    if (o != OP_NONE) {
      ktouched[a] = 1;
      ktouched[b] = 1;
    }
  }
}

constexpr u32 DEL_MARK = 0xFFFFFFFFu;

__global__ void k_emit_rowops(u32 U, const u32* seg_start, const u64* sk, const u8* op,
                              const u32* pos_del, const u32* pos_ins, u64 ins_base, u64* rkeys,
                              u32* rvals) {
  for (u64 j = blockIdx.x * (u64)blockDim.x + threadIdx.x; j < U; j += (u64)gridDim.x * blockDim.x) {
    u8 o = op[j];
    if (o != OP_DEL && o != OP_INS) continue;
    u64 key = sk[seg_start[j]];
    u32 a = (u32)(key >> 32), b = (u32)key;
    u64 p = (o == OP_DEL) ? pos_del[j] : ins_base + pos_ins[j];
    u32 val = (o == OP_DEL) ? DEL_MARK : (u32)j;
    rkeys[p] = ((u64)a << 32) | b;
    rvals[p] = val;
    rkeys[p + 1] = ((u64)b << 32) | a;
    rvals[p + 1] = val;
  }
}

__global__ void k_count_loops(u32 n, const u64* off, const u32* col, u32* total) {
  u32 local = 0;
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x) {
    u64 o0 = off[v], o1 = off[v + 1];
    u64 p = lower_bound_u32(col, o0, o1, (u32)v);
    while (p < o1 && col[p] == (u32)v) {
      ++local;
      ++p;
    }
  }
  if (local) atomicAdd(total, local);
}

// Existing self-loops are dropped by the reference's apply_delta
// (collect_canonical_edges keeps node < neighbor only, in_memory.rs:125).
__global__ void k_emit_loop_drops(u32 n, const u64* off, const u32* col, u64* rkeys, u32* rvals,
                                  u64 base, u64 limit, u32* counter, u8* ktouched, u32* err) {
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x) {
    u64 o0 = off[v], o1 = off[v + 1];
    u64 p = lower_bound_u32(col, o0, o1, (u32)v);
    u32 c = 0;
    while (p + c < o1 && col[p + c] == (u32)v) ++c;
    if (c) {
      u32 at = atomicAdd(counter, c);
      for (u32 i = 0; i < c; ++i) {
        if (base + at + i >= limit) {
          atomicAdd(err, 1u);
          break;
        }
        rkeys[base + at + i] = ((u64)v << 32) | (u32)v;
        rvals[base + at + i] = DEL_MARK;
      }
      ktouched[v] = 1;
    }
  }
}

__global__ void k_del_flags(const u32* rvals, u64 R, u32* flag) {
  for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t <= R; t += (u64)gridDim.x * blockDim.x)
    flag[t] = (t < R && rvals[t] == DEL_MARK) ? 1u : 0u;
}

__global__ void k_rowop_deg(const u64* rkeys, const u32* rvals, u64 R, int* ddeg, u8* touched) {
  for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < R; t += (u64)gridDim.x * blockDim.x) {
    u32 r = (u32)(rkeys[t] >> 32);
    atomicAdd(&ddeg[r], rvals[t] == DEL_MARK ? -1 : 1);
    touched[r] = 1;
  }
}

__global__ void k_new_degrees(u32 n, const u64* off, const int* ddeg, u64* nd) {
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v <= n; v += (u64)gridDim.x * blockDim.x)
    nd[v] = v < n ? (u64)((long long)(off[v + 1] - off[v]) + ddeg[v]) : 0ull;
}

// Untouched rows of the new CSR, copied by output position: each block takes
// COPY_CH consecutive output entries and finds the rows they span with two
// warp searches.  It stages those rows' new offsets, their shifts (old minus
// new offset) and touched flags in shared memory, maps every entry to its row
// there, and moves four entries per thread at a time.  Reads and writes
// stream; entries of touched rows are left to k_merge_rows.
constexpr u32 COPY_CH = 4096;
constexpr u32 COPY_ROWS = 1024;
constexpr u32 COPY_UNROLL = 4;

// Largest i in [lo, hi) with a[i] <= x, given a[lo] <= x (a ascending).
__device__ __forceinline__ u64 last_le_u64(const u64* a, u64 lo, u64 hi, u64 x) {
  while (hi - lo > 1) {
    const u64 mid = lo + (hi - lo) / 2;
    if (a[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// The same search by a whole warp: each step probes 32 evenly spaced
// positions lo + span·k/32 at once and keeps the interval between the last
// probe <= x and the next, so the span shrinks 32-fold per step.
__device__ __forceinline__ u64 warp_last_le_u64(const u64* a, u64 lo, u64 hi, u64 x) {
  const u32 lane = threadIdx.x & 31;
  while (hi - lo > 32) {
    const u64 span = hi - lo;
    const u64 p = lo + span * lane / 32;
    const u32 m = __ballot_sync(0xffffffffu, lane == 0 || a[p] <= x);
    const u32 j = (u32)__popc(m) - 1;  // probes 0..j are <= x
    const u64 nlo = lo + span * j / 32;
    hi = j == 31 ? hi : lo + span * (j + 1) / 32;
    lo = nlo;
  }
  const u64 p = lo + lane;
  const u32 m = __ballot_sync(0xffffffffu, p < hi && (lane == 0 || a[p] <= x));
  return lo + (u32)__popc(m) - 1;
}

__global__ void __launch_bounds__(256) k_copy_untouched(u32 n, const u64* off, const u32* col,
                                                        const double* w, const u64* noff,
                                                        u32* ncol, double* nw, const u8* touched,
                                                        u64 nnz_new) {
  __shared__ u64 s_noff[COPY_ROWS + 1];
  __shared__ u64 s_shift[COPY_ROWS];
  __shared__ u8 s_touched[COPY_ROWS];
  __shared__ u32 s_rb, s_re;
  const u32 wid = threadIdx.x >> 5;
  for (u64 q0 = (u64)blockIdx.x * COPY_CH; q0 < nnz_new; q0 += (u64)gridDim.x * COPY_CH) {
    const u64 q1 = q0 + COPY_CH < nnz_new ? q0 + COPY_CH : nnz_new;
    // rows r with noff[r] <= q < noff[r + 1]; noff[0] = 0 <= q0, noff[n] = nnz_new > q
    if (wid == 0) {
      const u64 rb = warp_last_le_u64(noff, 0, (u64)n + 1, q0);
      if ((threadIdx.x & 31) == 0) s_rb = (u32)rb;
    } else if (wid == 1) {
      const u64 re = warp_last_le_u64(noff, 0, (u64)n + 1, q1 - 1);
      if ((threadIdx.x & 31) == 0) s_re = (u32)re;
    }
    __syncthreads();
    const u32 rb = s_rb;
    const u32 nrow = s_re - rb + 1;  // re <= n - 1, so rb + nrow <= n
    const bool staged = nrow <= COPY_ROWS;
    if (staged)
      for (u32 x = threadIdx.x; x <= nrow; x += blockDim.x) {
        const u64 no = noff[rb + x];
        s_noff[x] = no;
        if (x < nrow) {
          s_shift[x] = off[rb + x] - no;  // modulo 2^64: src = q + shift
          s_touched[x] = touched[rb + x];
        }
      }
    __syncthreads();
    for (u64 qb = q0 + threadIdx.x; qb < q1; qb += COPY_UNROLL * blockDim.x) {
      u64 src[COPY_UNROLL];
      bool mv[COPY_UNROLL];
#pragma unroll
      for (u32 u = 0; u < COPY_UNROLL; ++u) {
        const u64 q = qb + (u64)u * blockDim.x;
        mv[u] = false;
        src[u] = 0;
        if (q < q1) {
          if (staged) {
            u32 lo = 0, hi = nrow;
            while (hi - lo > 1) {
              const u32 mid = (lo + hi) >> 1;
              if (s_noff[mid] <= q) lo = mid;
              else hi = mid;
            }
            mv[u] = !s_touched[lo];
            src[u] = q + s_shift[lo];
          } else {
            const u32 r = (u32)last_le_u64(noff, rb, (u64)rb + nrow, q);
            mv[u] = !touched[r];
            src[u] = off[r] + (q - noff[r]);
          }
        }
      }
      u32 c[COPY_UNROLL];
      double v[COPY_UNROLL];
#pragma unroll
      for (u32 u = 0; u < COPY_UNROLL; ++u)
        if (mv[u]) {
          c[u] = col[src[u]];
          v[u] = w[src[u]];
        }
#pragma unroll
      for (u32 u = 0; u < COPY_UNROLL; ++u)
        if (mv[u]) {
          const u64 q = qb + (u64)u * blockDim.x;
          ncol[q] = c[u];
          nw[q] = v[u];
        }
    }
    __syncthreads();
  }
}

// Row-operation range [rstart[r], rend[r]) of every row that has operations
// (row-operations sorted by (row, neighbour)).
__global__ void k_row_ranges(const u64* rkeys, u64 R, u32* rstart, u32* rend) {
  for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < R; t += (u64)gridDim.x * blockDim.x) {
    const u32 r = (u32)(rkeys[t] >> 32);
    if (t == 0 || (u32)(rkeys[t - 1] >> 32) != r) rstart[r] = (u32)t;
    if (t + 1 == R || (u32)(rkeys[t + 1] >> 32) != r) rend[r] = (u32)(t + 1);
  }
}

// Merge of the row slice [s0, s1) (chunks of 32 from the row start o0) of a
// touched row, by one warp (the row merge itself is described at
// k_merge_rows).  The state on entry is that of the operations
// consumed before the slice: p = first operation not consumed, drun / irun =
// deletes / inserts consumed, del_key / del_same = neighbour of the last
// consumed delete and the consumed deletes on it.  `row_end` marks the row's
// last slice, whose last chunk takes every remaining operation.
__device__ __forceinline__ void merge_slice(u64 o0, u64 s0, u64 s1, bool row_end, u64 no, u32 p,
                                            u32 b, u32 drun, u32 irun, u32 del_key,
                                            u32 del_same, const u32* col, const double* w,
                                            u32* ncol, double* nw, const u64* rkeys,
                                            const u32* rvals, const double* neww, u64 nnz_new,
                                            u32* err) {
  const u32 lane = threadIdx.x & 31;
  // operation tile [tb, tb + 32) in registers: neighbour, value (DEL_MARK
  // for a delete, else the index of the inserted weight)
  u32 tb = p;
  u32 tk = NONE32, tv = 0;
  if (tb + lane < b) {
    tk = (u32)rkeys[tb + lane];
    tv = rvals[tb + lane];
  }
  // entry chunk prefetched one ahead
  u32 c_n = s0 + lane < s1 ? col[s0 + lane] : NONE32;
  double w_n = s0 + lane < s1 ? w[s0 + lane] : 0.0;
  for (u64 base = s0;; base += 32) {
    const bool chunk_last = base + 32 >= s1;
    const bool last = chunk_last && row_end;  // the row's last chunk takes every remaining op
    const u64 q = base + lane;
    const bool valid = q < s1;
    const u32 c = c_n;
    const double wv = w_n;
    if (!chunk_last) {
      const u64 qn = q + 32;
      c_n = qn < s1 ? col[qn] : NONE32;
      w_n = qn < s1 ? w[qn] : 0.0;
    }
    const u32 vmask = __ballot_sync(0xffffffffu, valid);
    const u32 c_last = vmask ? __shfl_sync(0xffffffffu, c, 31 - __clz(vmask)) : 0u;
    const u32 d0 = drun, i0 = irun;
    u32 dl = 0, il = 0;
    // the two copies of a deleted self-loop may straddle two chunks: the
    // earlier chunk consumed their deletes
    bool deleted = valid && del_key != NONE32 && c == del_key;
    while (p < b) {
      const u32 o = p - tb;  // first unconsumed lane of the tile
      const bool ok = tb + lane < b && lane >= o;
      const u32 m = __ballot_sync(0xffffffffu, ok && (last || tk <= c_last));
      const u32 cnt = __popc(m);  // lanes o .. o+cnt-1 (operations are sorted)
      if (cnt) {
        const u32 hiL = o + cnt;
        const u32 delm = __ballot_sync(0xffffffffu, tv == DEL_MARK) & m;
        // Entries: the consumed operations below c (lower bound of c among
        // the tile's keys) and whether c itself is deleted.
        u32 lo = o, hi = hiL;
#pragma unroll
        for (int it = 0; it < 6; ++it) {
          const u32 mid = (lo + hi) >> 1;
          const u32 km = __shfl_sync(0xffffffffu, tk, mid & 31);
          if (lo < hi) {
            if (km < c) lo = mid + 1;
            else hi = mid;
          }
        }
        const u32 ltm = m & (lo >= 32 ? 0xffffffffu : ((1u << lo) - 1u));
        dl += __popc(ltm & delm);
        il += __popc(ltm & ~delm);
        const u32 kp = __shfl_sync(0xffffffffu, tk, lo & 31);
        const u32 vp = __shfl_sync(0xffffffffu, tv, lo & 31);
        if (valid && lo < hiL && kp == c && vp == DEL_MARK) deleted = true;
        // Inserts: lower bound among the chunk's entries (padded with
        // NONE32), earlier deletes below the key and earlier inserts.
        u32 lo2 = 0, hi2 = 32;
#pragma unroll
        for (int it = 0; it < 6; ++it) {
          const u32 mid = (lo2 + hi2) >> 1;
          const u32 cm = __shfl_sync(0xffffffffu, c, mid & 31);
          if (lo2 < hi2) {
            if (cm < tk) lo2 = mid + 1;
            else hi2 = mid;
          }
        }
        const u32 grp = __match_any_sync(0xffffffffu, tk) & m;
        const u32 before = (1u << lane) - 1u;
        const bool ins = ((m >> lane) & 1u) && tv != DEL_MARK;
        if (ins) {
          const u32 dlt = drun + __popc(delm & before) - __popc(grp & delm & before) -
                          (del_key == tk ? del_same : 0u);
          const u64 out = no + (base + lo2 - o0) - dlt + irun + __popc(m & ~delm & before);
          if (out >= nnz_new) {
            atomicAdd(err, 1u);
          } else {
            ncol[out] = tk;
            nw[out] = neww[tv];
          }
        }
        if (delm) {
          const u32 ld = 31 - __clz(delm);
          const u32 kd = __shfl_sync(0xffffffffu, tk, ld);
          const u32 same = __popc(__shfl_sync(0xffffffffu, grp, ld) & delm);
          del_same = (del_key == kd) ? del_same + same : same;
          del_key = kd;
        }
        drun += __popc(delm);
        irun += cnt - __popc(delm);
      }
      p += cnt;
      if (o + cnt < 32 || p >= b) break;
      // the whole tile was consumed: load the next one
      tb = p;
      tk = NONE32;
      tv = 0;
      if (tb + lane < b) {
        tk = (u32)rkeys[tb + lane];
        tv = rvals[tb + lane];
      }
    }
    if (valid && !deleted) {
      const u64 out = no + (q - o0) - (d0 + dl) + (i0 + il);
      if (out >= nnz_new) {
        atomicAdd(err, 1u);
      } else {
        ncol[out] = c;
        nw[out] = wv;
      }
    }
    if (chunk_last) break;
  }
}

// Touched rows, merged with their sorted row-operations, so the output row is
// again sorted by neighbour id: deleted entries are skipped, every surviving
// entry moves by (inserts before it) - (deletes before it), and an insert
// lands at its lower bound in the old row, after the earlier inserts and
// before the entries it precedes.  A warp walks the row in chunks of 32 and
// consumes, per chunk, the operations whose neighbour is not above the
// chunk's last one (all of them in the row's last chunk), 32 operations at a
// time with bisections over lanes.  A self-loop is stored twice in its row and
// its operations come in pairs; operations on one neighbour come deletes
// first (a dropped self-loop replaced by an inserted one).
//
// Rows longer than MERGE_LONG go to `long_rows` for k_merge_long.
constexpr u64 MERGE_LONG = 512;

__global__ void k_merge_rows(u32 n, const u64* off, const u32* col, const double* w,
                             const u64* noff, u32* ncol, double* nw, const u8* touched,
                             const u64* rkeys, const u32* rvals, const u32* rstart,
                             const u32* rend, const double* neww, u64 nnz_new, u32* err,
                             u32* long_rows, u32* nlong) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 r = warp; r < n; r += nwarps) {
    if (!touched[r]) continue;
    const u64 o0 = off[r], o1 = off[r + 1];
    if (o1 - o0 > MERGE_LONG) {
      if (lane == 0) long_rows[atomicAdd(nlong, 1u)] = (u32)r;
      continue;
    }
    merge_slice(o0, o0, o1, true, noff[r], rstart[r], rend[r], 0, 0, NONE32, 0, col, w, ncol, nw,
                rkeys, rvals, neww, nnz_new, err);
  }
}

// Long touched rows: a block per row, its warps on consecutive slices of
// whole chunks.  A warp rebuilds the state at its slice start from the
// operations whose neighbour is not above the entry before the slice (a
// bisection, and the delete prefix of the sorted operations).
__global__ void __launch_bounds__(256) k_merge_long(const u32* long_rows, const u32* nlong,
                                                    const u64* off, const u32* col,
                                                    const double* w, const u64* noff, u32* ncol,
                                                    double* nw, const u64* rkeys,
                                                    const u32* rvals, const u32* rstart,
                                                    const u32* rend, const u32* delpre,
                                                    const double* neww, u64 nnz_new, u32* err) {
  const u32 lane = threadIdx.x & 31;
  const u32 wib = threadIdx.x >> 5;
  const u32 nw_ = blockDim.x >> 5;
  const u32 cnt = *nlong;
  for (u32 t = blockIdx.x; t < cnt; t += gridDim.x) {
    const u32 r = long_rows[t];
    const u64 o0 = off[r], o1 = off[r + 1];
    const u64 chunks = (o1 - o0 + 31) / 32;  // > MERGE_LONG / 32 >= warps per block
    const u64 c0 = chunks * wib / nw_, c1 = chunks * (wib + 1) / nw_;
    const u64 s0 = o0 + 32 * c0;
    const u64 s1 = (o0 + 32 * c1 < o1) ? o0 + 32 * c1 : o1;
    const u32 a = rstart[r], b = rend[r];
    u32 p = a, drun = 0, irun = 0, del_key = NONE32, del_same = 0;
    if (s0 > o0) {
      // operations consumed before the slice: neighbour <= cprev = col[s0 - 1]
      const u32 cprev = col[s0 - 1];
      u32 lo = a, hi = b;
      while (lo < hi) {
        const u32 mid = (lo + hi) >> 1;
        if ((u32)rkeys[mid] <= cprev) lo = mid + 1;
        else hi = mid;
      }
      p = lo;
      drun = delpre[p] - delpre[a];
      irun = (p - a) - drun;
      // Only deletes on cprev itself matter from here on (a self-loop whose
      // two copies the slice boundary separates): entries of this slice and
      // the operations still to come are all >= cprev.
      u32 x = p;
      while (x > a && (u32)rkeys[x - 1] == cprev) --x;
      for (; x < p; ++x)
        if (rvals[x] == DEL_MARK) ++del_same;
      if (del_same) del_key = cprev;
    }
    merge_slice(o0, s0, s1, c1 == chunks, noff[r], p, b, drun, irun, del_key, del_same, col, w,
                ncol, nw, rkeys, rvals, neww, nnz_new, err);
  }
}

// Row sums in CSR order (hit_leiden.rs:1063), left to right: the exact
// rounding of the reference for any weights (warp per row, ordered fold).
// `flags` (if set) restricts the rows to those flagged.  Rows of RUN_FOLD_MIN
// or more entries are listed for k_row_sum_runs.
__global__ void k_row_sum_serial(const u32* rows, u32 nr, const u64* off, const double* w,
                                 double* k, const u8* flags, u32* longl, u32* longn) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 i = warp; i < nr; i += nwarps) {
    u32 v = rows ? rows[i] : (u32)i;
    if (flags && !flags[v]) continue;
    const u64 a = off[v], b = off[v + 1];
    if (b - a >= RUN_FOLD_MIN) {
      fold_defer(longl, longn, v);
      continue;
    }
    double s = warp_ordered_sum(a, b, 0.0, [&](u64 p) { return w[p]; },
                                [](u64) { return true; });
    if (lane == 0) k[v] = s;
  }
}

// The long rows listed by k_row_sum_serial, folded in runs (the same bits).
__global__ void k_row_sum_runs(const u32* longl, const u32* longn, const u64* off,
                               const double* w, double* k) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  const u32 nl = *longn;
  for (u64 j = warp; j < nl; j += nwarps) {
    const u32 v = longl[j];
    double s = warp_fold_runs(off[v], off[v + 1], 0.0, w);
    if (lane == 0) k[v] = s;
  }
}

// Left-to-right sums of the segments [off[i], off[i+1]) of x from `init`:
// PATH 0 is the library's pair (short segments here, long ones listed for
// k_seq_sums_runs), 1 folds every segment in runs, 2 none.
template <int PATH>
__global__ void k_seq_sums(u32 nseg, const u64* off, const double* x, double init, double* out,
                           u32* longl, u32* longn) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 i = warp; i < nseg; i += nwarps) {
    const u64 a = off[i], b = off[i + 1];
    double s;
    if constexpr (PATH == 1) {
      s = warp_fold_runs(a, b, init, x);
    } else {
      if (PATH == 0 && b - a >= RUN_FOLD_MIN) {
        fold_defer(longl, longn, (u32)i);
        continue;
      }
      s = warp_ordered_sum(a, b, init, [&](u64 p) { return x[p]; }, [](u64) { return true; });
    }
    if (lane == 0) out[i] = s;
  }
}

__global__ void k_seq_sums_runs(const u32* longl, const u32* longn, const u64* off,
                                const double* x, double init, double* out) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  const u32 nl = *longn;
  for (u64 j = warp; j < nl; j += nwarps) {
    const u32 i = longl[j];
    double s = warp_fold_runs(off[i], off[i + 1], init, x);
    if (lane == 0) out[i] = s;
  }
}

FoldList fold_list(Engine& E, u64 total, u32 nseg) {
  Scratch& S = E.sc;
  u64 cap = total / RUN_FOLD_MIN + 1;
  if (cap > nseg) cap = nseg ? nseg : 1;
  S.foldseg.ensure(E.mem, cap);
  S.foldcnt.ensure(E.mem, 1);
  HL_CUDA(cudaMemsetAsync(S.foldcnt.p, 0, sizeof(u32), E.stream));
  return FoldList{S.foldseg.p, S.foldcnt.p};
}

void seq_sums(Engine& E, u32 nseg, const u64* off, const double* x, double init, int path,
              double* out) {
  if (!nseg) return;
  const u32 grid = grid_for((u64)nseg * 32);
  if (path == 1) {
    ++E.nlaunch, k_seq_sums<1><<<grid, 256, 0, E.stream>>>(nseg, off, x, init, out, nullptr,
                                                            nullptr);
  } else if (path == 2) {
    ++E.nlaunch, k_seq_sums<2><<<grid, 256, 0, E.stream>>>(nseg, off, x, init, out, nullptr,
                                                            nullptr);
  } else {
    // the total is only known on the device: room for every segment
    FoldList fl = fold_list(E, (u64)nseg * RUN_FOLD_MIN, nseg);
    ++E.nlaunch, k_seq_sums<0><<<grid, 256, 0, E.stream>>>(nseg, off, x, init, out, fl.seg,
                                                            fl.cnt);
    ++E.nlaunch, k_seq_sums_runs<<<FOLD_BLOCKS, 256, 0, E.stream>>>(fl.seg, fl.cnt, off, x, init,
                                                                  out);
  }
  HL_LAUNCH_CHECK();
}

// Ordered row sums of the flagged rows (all rows without flags): the short
// rows in k_row_sum_serial, the long ones in k_row_sum_runs.
static void row_sums_ordered(Engine& E, Level& L, const u8* flags) {
  const u32 n = L.g.n;
  FoldList fl = fold_list(E, L.g.nnz, n);
  ++E.nlaunch, k_row_sum_serial<<<grid_for((u64)n * 32), 256, 0, E.stream>>>(
      nullptr, n, L.g.off.p, L.g.w.p, L.k.p, flags, fl.seg, fl.cnt);
  ++E.nlaunch, k_row_sum_runs<<<FOLD_BLOCKS, 256, 0, E.stream>>>(fl.seg, fl.cnt, L.g.off.p,
                                                                 L.g.w.p, L.k.p);
}

// Warp-parallel row sums; only used when every weight is integral, where any
// summation order gives the same bits.
__global__ void k_row_sum_warp(const u32* rows, u32 nr, const u64* off, const double* w,
                               double* k, const u8* flags = nullptr) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 i = warp; i < nr; i += nwarps) {
    u32 v = rows ? rows[i] : (u32)i;
    if (flags && !flags[v]) continue;
    double s = 0.0;
    for (u64 p = off[v] + lane; p < off[v + 1]; p += 32) s += w[p];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) k[v] = s;
  }
}


// Fixed-shape pairwise sum: tiles of 1024 (+0.0 padded) folded by stride
// halving; repeated on the tile sums until one value remains.
__global__ void k_tree_tile(const double* x, u64 n, double* out) {
  __shared__ double s[1024];
  u64 base = (u64)blockIdx.x * 1024;
  for (u32 i = threadIdx.x; i < 1024; i += blockDim.x) {
    u64 idx = base + i;
    s[i] = idx < n ? x[idx] : 0.0;
  }
  __syncthreads();
  for (u32 st = 512; st >= 1; st >>= 1) {
    for (u32 i = threadIdx.x; i < st; i += blockDim.x) s[i] = __dadd_rn(s[i], s[i + st]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

double tree_sum(Engine& E, const double* x, u64 n) {
  if (n == 0) return 0.0;
  u64 tiles = (n + 1023) / 1024;
  E.sc.red.ensure(E.mem, tiles + 1);
  E.sc.red2.ensure(E.mem, (tiles + 1023) / 1024 + 1);
  const double* src = x;
  double* a = E.sc.red.p;
  double* b = E.sc.red2.p;
  u64 cur = n;
  while (true) {
    u64 t = (cur + 1023) / 1024;
    ++E.nlaunch, k_tree_tile<<<(u32)t, 256, 0, E.stream>>>(src, cur, a);
    HL_LAUNCH_CHECK();
    if (t == 1) break;
    src = a;
    cur = t;
    std::swap(a, b);
  }
  return E.read_f64(a);
}

// Rows whose flag is set (no list, so no count to read back first).
static void recompute_flagged_rows(Engine& E, Level& L, const u8* flags) {
  const u32 n = L.g.n;
  if (!n) return;
  cudaEvent_t ev = E.kt_begin();
  if (E.integral)
    ++E.nlaunch, k_row_sum_warp<<<grid_for((u64)n * 32), 256, 0, E.stream>>>(
        nullptr, n, L.g.off.p, L.g.w.p, L.k.p, flags);
  else
    row_sums_ordered(E, L, flags);
  HL_LAUNCH_CHECK();
  E.kt_end(KT_ROW_SUMS, ev);
}

void recompute_all_degrees(Engine& E, Level& L) {
  u32 n = L.g.n;
  if (n) {
    if (E.integral)
      ++E.nlaunch, k_row_sum_warp<<<grid_for((u64)n * 32), 256, 0, E.stream>>>(nullptr, n, L.g.off.p, L.g.w.p,
                                                                   L.k.p);
    else
      row_sums_ordered(E, L, nullptr);
    HL_LAUNCH_CHECK();
  }
  L.tw = tree_sum(E, L.k.p, n);
}

struct FlagToIndex {
  const u8* f;
  __host__ __device__ bool operator()(const u32& i) const { return f[i] != 0; }
};

void apply_delta(Engine& E, Level& L, const DevEdges& b, u32 new_n, bool keep_loops) {
  Scratch& S = E.sc;
  cudaStream_t st = E.stream;
  if (new_n > L.g.n) graph_grow_nodes(E, L, new_n);
  const u32 n = L.g.n;
  const bool drop_loops = !keep_loops && L.g.self_loop_entries > 0;
  if (b.k == 0 && !drop_loops) return;
  const u64 k = b.k;

  S.ktouched.ensure(E.mem, n ? n : 1);
  HL_CUDA(cudaMemsetAsync(S.ktouched.p, 0, n ? n : 1, st));
  S.cnt.ensure(E.mem, 16);
  HL_CUDA(cudaMemsetAsync(S.cnt.p, 0, 16 * sizeof(u32), st));  // [0] ins loops [1] del loops [2] drops

  u32 U = 0;
  cudaEvent_t ev_ds = E.kt_begin();
  if (k) {
    S.keys.ensure(E.mem, k);
    S.keys2.ensure(E.mem, k);
    S.idx.ensure(E.mem, k);
    S.idx2.ensure(E.mem, k);
    S.segid.ensure(E.mem, k);
    S.seg_start.ensure(E.mem, k + 1);
    S.rowlist.ensure(E.mem, k);
    ++E.nlaunch, k_delta_keys<<<grid_for(k), 256, 0, st>>>(b.u, b.v, k, S.keys.p, S.idx.p);
    HL_LAUNCH_CHECK();
    u64* kin = S.keys.p;
    u64* kout = S.keys2.p;
    u32* vin = S.idx.p;
    u32* vout = S.idx2.p;
    cub_run(E, [&](void* t, size_t& bytes) {
      // keys (u << 32) | v with u, v < n
      return cub::DeviceRadixSort::SortPairs(t, bytes, kin, kout, vin, vout, (int64_t)k, 0,
                                             32 + bits_for(n ? n - 1 : 0), st);
    });
    ++E.nlaunch, k_heads<<<grid_for(k), 256, 0, st>>>(kout, k, S.rowlist.p);
    HL_LAUNCH_CHECK();
    u32* head = S.rowlist.p;
    u32* segid = S.segid.p;
    cub_run(E, [&](void* t, size_t& bytes) {
      return cub::DeviceScan::ExclusiveSum(t, bytes, head, segid, (int64_t)k, st);
    });
    ++E.nlaunch, k_seg_start<<<grid_for(k), 256, 0, st>>>(head, segid, k, S.seg_start.p);
    HL_LAUNCH_CHECK();
    u32 lh[2];
    E.read_u32s({segid + (k - 1), head + (k - 1)}, lh);
    U = lh[0] + lh[1];

    S.op.ensure(E.mem, U);
    S.neww.ensure(E.mem, U);
    S.nops_del.ensure(E.mem, U + 1);
    S.nops_ins.ensure(E.mem, U + 1);
    S.pos_del.ensure(E.mem, U + 1);
    S.pos_ins.ensure(E.mem, U + 1);
    ++E.nlaunch, k_resolve<<<grid_for(U), 256, 0, st>>>(U, S.seg_start.p, k, kout, vout, b.w, L.g.off.p,
                                           L.g.col.p, L.g.w.p, keep_loops, S.op.p, S.neww.p,
                                           S.ktouched.p, S.nops_del.p, S.nops_ins.p, S.cnt.p);
    HL_LAUNCH_CHECK();
    HL_CUDA(cudaMemsetAsync(S.nops_del.p + U, 0, sizeof(u32), st));
    HL_CUDA(cudaMemsetAsync(S.nops_ins.p + U, 0, sizeof(u32), st));
    u32* nd = S.nops_del.p;
    u32* pd = S.pos_del.p;
    u32* ni = S.nops_ins.p;
    u32* pi = S.pos_ins.p;
    cub_run(E, [&](void* t, size_t& bytes) {
      return cub::DeviceScan::ExclusiveSum(t, bytes, nd, pd, (int64_t)U + 1, st);
    });
    cub_run(E, [&](void* t, size_t& bytes) {
      return cub::DeviceScan::ExclusiveSum(t, bytes, ni, pi, (int64_t)U + 1, st);
    });
  }
  E.kt_end(KT_DELTA_SORT, ev_ds);
  u64 n_del_keys = 0, n_ins = 0;
  if (U) {
    u32 di[2];
    E.read_u32s({S.pos_del.p + U, S.pos_ins.p + U}, di);
    n_del_keys = di[0];
    n_ins = di[1];
  }

  // Existing self-loops to drop (reference behaviour) — counted first.
  u64 n_drop = 0;
  if (drop_loops) {
    HL_CUDA(cudaMemsetAsync(S.cnt.p + 3, 0, sizeof(u32), st));
    ++E.nlaunch, k_count_loops<<<grid_for(n), 256, 0, st>>>(n, L.g.off.p, L.g.col.p, S.cnt.p + 3);
    HL_LAUNCH_CHECK();
    n_drop = E.read_u32(S.cnt.p + 3);
  }
  u64 R = n_del_keys + n_drop + n_ins;

  if (R == 0) {
    // Weight updates only: no structural change.
    if (U) {
      recompute_flagged_rows(E, L, S.ktouched.p);
      L.tw = tree_sum(E, L.k.p, n);
    }
    return;
  }

  S.rkeys.ensure(E.mem, R);
  S.rkeys2.ensure(E.mem, R);
  S.rvals.ensure(E.mem, R);
  S.rvals2.ensure(E.mem, R);
  if (U)
    ++E.nlaunch, k_emit_rowops<<<grid_for(U), 256, 0, st>>>(U, S.seg_start.p, S.keys2.p, S.op.p, S.pos_del.p,
                                               S.pos_ins.p, n_del_keys + n_drop, S.rkeys.p,
                                               S.rvals.p);
  if (drop_loops && n_drop)
    ++E.nlaunch, k_emit_loop_drops<<<grid_for(n), 256, 0, st>>>(n, L.g.off.p, L.g.col.p, S.rkeys.p, S.rvals.p,
                                                   n_del_keys, n_del_keys + n_drop, S.cnt.p + 2,
                                                   S.ktouched.p, S.cnt.p + 4);
  HL_LAUNCH_CHECK();
  {
    u64* kin = S.rkeys.p;
    u64* kout = S.rkeys2.p;
    u32* vin = S.rvals.p;
    u32* vout = S.rvals2.p;
    cub_run(E, [&](void* t, size_t& bytes) {
      // keys (row << 32) | neighbour with both < n
      return cub::DeviceRadixSort::SortPairs(t, bytes, kin, kout, vin, vout, (int64_t)R, 0,
                                             32 + bits_for(n ? n - 1 : 0), st);
    });
  }
  require(R < 0xFFFFFFFFull, "too many row operations in one batch");
  // row-operation range of every row that has operations
  S.delpre.ensure(E.mem, n ? n : 1);
  S.inspre.ensure(E.mem, n ? n : 1);
  ++E.nlaunch, k_row_ranges<<<grid_for(R), 256, 0, st>>>(S.rkeys2.p, R, S.delpre.p, S.inspre.p);
  // deletes before every operation (for the long-row merge's slice starts)
  S.opdel.ensure(E.mem, R + 1);
  S.opdelpre.ensure(E.mem, R + 1);
  ++E.nlaunch, k_del_flags<<<grid_for(R + 1), 256, 0, st>>>(S.rvals2.p, R, S.opdel.p);
  HL_LAUNCH_CHECK();
  {
    u32* a = S.opdel.p;
    u32* o = S.opdelpre.p;
    cub_run(E, [&](void* t, size_t& bytes) {
      return cub::DeviceScan::ExclusiveSum(t, bytes, a, o, (int64_t)R + 1, st);
    });
  }
  S.ddeg.ensure(E.mem, n ? n : 1);
  S.touched.ensure(E.mem, n ? n : 1);
  HL_CUDA(cudaMemsetAsync(S.ddeg.p, 0, sizeof(int) * (n ? n : 1), st));
  HL_CUDA(cudaMemsetAsync(S.touched.p, 0, n ? n : 1, st));
  ++E.nlaunch, k_rowop_deg<<<grid_for(R), 256, 0, st>>>(S.rkeys2.p, S.rvals2.p, R, S.ddeg.p, S.touched.p);
  S.newoff.ensure(E.mem, (size_t)n + 1);
  ++E.nlaunch, k_new_degrees<<<grid_for((u64)n + 1), 256, 0, st>>>(n, L.g.off.p, S.ddeg.p, S.newoff.p);
  HL_LAUNCH_CHECK();
  {
    u64* a = S.newoff.p;
    cub_run(E, [&](void* t, size_t& bytes) {
      return cub::DeviceScan::ExclusiveSum(t, bytes, a, a, (int64_t)n + 1, st);
    });
  }
  u64 nnz_new = E.read_u64(S.newoff.p + n);
  DevGraph& G = L.g;
  DBuf<u32>& ncol = G.col2;
  DBuf<double>& nw = G.w2;
  ncol.ensure(E.mem, nnz_new ? nnz_new : 1);
  nw.ensure(E.mem, nnz_new ? nnz_new : 1);
  cudaEvent_t cev = E.kt_begin();
  if (nnz_new)
    ++E.nlaunch, k_copy_untouched<<<grid_for((nnz_new + COPY_CH - 1) / COPY_CH * 256), 256, 0, st>>>(
        n, G.off.p, G.col.p, G.w.p, S.newoff.p, ncol.p, nw.p, S.touched.p, nnz_new);
  E.kt_end(KT_COPY_ROWS, cev);
  cudaEvent_t kev = E.kt_begin();
  if (n) {
    S.ovf.ensure(E.mem, n);
    S.ovf_cnt.ensure(E.mem, 4);
    HL_CUDA(cudaMemsetAsync(S.ovf_cnt.p, 0, sizeof(u32), st));
    ++E.nlaunch, k_merge_rows<<<grid_for((u64)n * 32), 256, 0, st>>>(
        n, G.off.p, G.col.p, G.w.p, S.newoff.p, ncol.p, nw.p, S.touched.p, S.rkeys2.p, S.rvals2.p,
        S.delpre.p, S.inspre.p, S.neww.p, nnz_new, S.cnt.p + 4, S.ovf.p, S.ovf_cnt.p);
    ++E.nlaunch, k_merge_long<<<148 * 2, 256, 0, st>>>(
        S.ovf.p, S.ovf_cnt.p, G.off.p, G.col.p, G.w.p, S.newoff.p, ncol.p, nw.p, S.rkeys2.p,
        S.rvals2.p, S.delpre.p, S.inspre.p, S.opdelpre.p, S.neww.p, nnz_new, S.cnt.p + 4);
  }
  HL_LAUNCH_CHECK();
  E.kt_end(KT_MERGE_ROWS, kev);
  // old and new offsets, touched flags, old and new (col, w) entries
  E.kagg[KT_MERGE_ROWS].bytes += 16ull * ((u64)n + 1) + n + 12ull * (G.nnz + nnz_new);
  u32 ce[3];  // merge errors, inserted and deleted self-loops
  E.read_u32s({S.cnt.p + 4, S.cnt.p + 0, S.cnt.p + 1}, ce);
  if (ce[0] != 0)
    throw Error(HL_ERR_CUDA, "internal error: CSR merge produced an out-of-range position");
  G.col.swap(ncol);
  G.w.swap(nw);
  G.off.swap(S.newoff);
  G.nnz = nnz_new;
  {
    u32 ins_loops = ce[1];
    u32 del_loops = ce[2];
    if (drop_loops)
      G.self_loop_entries = 2ull * ins_loops;
    else
      G.self_loop_entries = G.self_loop_entries + 2ull * ins_loops - 2ull * del_loops;
  }
  // Degrees of every row whose weights changed, then 2m.
  recompute_flagged_rows(E, L, S.ktouched.p);
  L.tw = tree_sum(E, L.k.p, n);
}

}  // namespace hl
