// refine.cu — inc-refinement, throughput mode (hit_leiden.rs:1265-1390,
// :1554-1637; throughput.rs:239-359).
//
//  1. Sub-communities holding a K vertex are split into connected components
//     over edges whose ends share the sub-community (and, in the multi-level
//     mode, the community).  Components come from a lock-free union-find that
//     always hooks the larger root under the smaller, so a root is its
//     component's minimum vertex — the BFS start the reference would use.
//  2. The largest component keeps the id; on equal sizes the last one in
//     discovery order (largest minimum vertex) wins, as Rust's max_by_key
//     does.  The others get max(s)+1, +2, … in (sub-community, minimum vertex)
//     order.
//  3. T-filter: a candidate sub-community S is blocked when
//     ΔQ(S→∅) = -w(S,C)/2m + γ d_S (d_C - d_S)/(2m)^2 > 1e-9.
//  4. Jacobi singleton merge: every refined singleton evaluates its best
//     same-community neighbour sub-community on the snapshot; all positive
//     moves are applied together.
#include "hl_engine.cuh"

namespace hl {

static inline u32 grid_for(u64 n, u32 block = 256) {
  u64 g = (n + block - 1) / block;
  if (g > 148u * 64u) g = 148u * 64u;
  return g ? (u32)g : 1u;
}

void run_eval(Engine& E, int kind, const u32* verts, u32 nv, const Level& L, const u32* s,
              const double* d, const u8* blocked, bool allow_empty, u32* out_to, double* out_gain,
              unsigned long long* traversed);

__global__ void k_mark_affected_sc(const u8* affected, const u32* s, u32 n, u8* affsc) {
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x)
    if (affected[v]) affsc[s[v]] = 1;
}

__device__ __forceinline__ u32 uf_find(u32* par, u32 x) {
  u32 p = par[x];
  while (p != x) {
    u32 gp = par[p];
    if (gp != p) par[x] = gp;  // path halving (always an ancestor)
    x = p;
    p = gp;
  }
  return x;
}

__device__ __forceinline__ void uf_unite(u32* par, u32 a, u32 b) {
  while (true) {
    a = uf_find(par, a);
    b = uf_find(par, b);
    if (a == b) return;
    u32 lo = a < b ? a : b, hi = a < b ? b : a;
    if (atomicCAS(&par[hi], hi, lo) == hi) return;
  }
}

__global__ void k_uf_edges(u32 n, const u64* off, const u32* col, const u32* s, const u32* f,
                           const u8* affsc, bool same_f, u32* par) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 v = warp; v < n; v += nwarps) {
    u32 sv = s[v];
    if (!affsc[sv]) continue;
    u32 fv = f[v];
    const u64 o1 = off[v + 1];
    // each undirected edge once (self-loops irrelevant): neighbours above v,
    // four entries per lane in flight
    for (u64 p0 = lower_bound_u32(col, off[v], o1, (u32)v + 1) + lane; p0 < o1; p0 += 128) {
      u32 nb[4], sn[4], fn[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) nb[j] = p0 + 32 * j < o1 ? col[p0 + 32 * j] : NONE32;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (nb[j] != NONE32) {
          sn[j] = s[nb[j]];
          fn[j] = same_f ? f[nb[j]] : fv;
        }
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (nb[j] != NONE32 && sn[j] == sv && fn[j] == fv) uf_unite(par, (u32)v, nb[j]);
    }
  }
}

// Every union is done: the forest no longer changes, so each vertex finds its
// root read-only (no path compression, which would race with the other
// threads' walks) and writes it to `root`.
__global__ void k_uf_final(u32 n, const u32* s, const u8* affsc, const u32* par, u32* root,
                           u32* csize) {
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x) {
    if (!affsc[s[v]]) continue;
    u32 r = (u32)v;
    while (par[r] != r) r = par[r];
    root[v] = r;
    atomicAdd(&csize[r], 1u);
  }
}

__global__ void k_keep(u32 n, const u32* s, const u8* affsc, const u32* par, const u32* csize,
                       unsigned long long* keep) {
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x) {
    if (!affsc[s[v]] || par[v] != v) continue;
    atomicMax(&keep[s[v]], ((unsigned long long)csize[v] << 32) | (u32)v);
  }
}

__global__ void k_split_roots(u32 n, const u32* s, const u8* affsc, const u32* par,
                              const unsigned long long* keep, u8* flag, u64* key) {
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x) {
    bool nk = affsc[s[v]] && par[v] == v && (u32)keep[s[v]] != (u32)v;
    flag[v] = nk ? 1 : 0;
    key[v] = ((u64)s[v] << 32) | (u32)v;
  }
}

__global__ void k_gather_keys(const u32* roots, u32 m, const u64* key, u64* out) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < m; i += (u64)gridDim.x * blockDim.x)
    out[i] = key[roots[i]];
}

__global__ void k_assign_newid(const u64* sorted, u32 m, u32 base, u32* newid, u32* origin_new,
                               u32* origin_old) {
  for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < m; t += (u64)gridDim.x * blockDim.x) {
    u32 r = (u32)sorted[t];
    newid[r] = base + (u32)t;
    origin_new[t] = base + (u32)t;
    origin_old[t] = (u32)(sorted[t] >> 32);
  }
}

__global__ void k_apply_split(u32 n, u32* s, const u8* affsc_snapshot, const u32* par,
                              const u8* nkflag, const u32* newid, u8* refined) {
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x) {
    u32 sv = s[v];
    if (!affsc_snapshot[sv]) continue;
    u32 r = par[v];
    if (nkflag[r]) {
      s[v] = newid[r];
      refined[v] = 1;
    }
  }
}

__global__ void k_not_identity(u32 n, const u32* s, u32* bad) {
  u32 local = 0;
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x)
    if (s[v] != (u32)v) ++local;
  if (local) atomicAdd(bad, local);
}

__global__ void k_refine_all_if_identity(u32 n, const u32* not_identity, u8* refined) {
  if (*not_identity) return;
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x)
    refined[v] = 1;
}

__global__ void k_sizes(u32 n, const u32* s, u32* sizes) {
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x)
    atomicAdd(&sizes[s[v]], 1u);
}

__global__ void k_singletons(const u32* rs, u32 nr, const u32* s, const u32* sizes, u8* flag) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < nr; i += (u64)gridDim.x * blockDim.x)
    flag[i] = sizes[s[rs[i]]] == 1 ? 1 : 0;
}

// Candidate sub-communities of the T-filter (hit_leiden.rs:1567-1586).
__global__ void k_t_candidates(const u32* single, u32 ns, const u64* off, const u32* col,
                               const u32* f, const u32* s, u8* cand) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 i = warp; i < ns; i += nwarps) {
    u32 v = single[i];
    u32 fv = f[v], sv = s[v];
    const u64 o1 = off[v + 1];
    for (u64 p0 = off[v] + lane; p0 < o1; p0 += 128) {
      u32 nb[4], fn[4], sn[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) nb[j] = p0 + 32 * j < o1 ? col[p0 + 32 * j] : NONE32;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (nb[j] != NONE32) {
          fn[j] = f[nb[j]];
          sn[j] = s[nb[j]];
        }
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (nb[j] != NONE32 && fn[j] == fv && sn[j] != sv) cand[sn[j]] = 1;
    }
  }
}

__global__ void k_min_member(u32 n, const u32* s, const u8* cand, u32* minmem) {
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x)
    if (cand[s[v]]) atomicMin(&minmem[s[v]], (u32)v);
}

// w(S, C_parent) summed in any order, with the number of terms.  The T-filter
// only needs the side of its threshold on which the ordered sum falls, and
// the any-order sum plus a rounding-error bound decides that for almost every
// S (k_blocked_bounds).  A warp per member row; rows longer than LONG_ROW go to
// a list that k_wsp_any_long covers with a whole block per row.
constexpr u32 LONG_ROW = 4096;

__device__ __forceinline__ void wsp_row_part(u64 a, u64 b, u64 step, const u32* col,
                                             const double* w, const u32* f, u32 parent,
                                             double& x, unsigned long long& c) {
  u64 p = a;
  for (; p + 3 * step < b; p += 4 * step) {
    const u32 c0 = col[p], c1 = col[p + step], c2 = col[p + 2 * step], c3 = col[p + 3 * step];
    const double w0 = w[p], w1 = w[p + step], w2 = w[p + 2 * step], w3 = w[p + 3 * step];
    const u32 f0 = f[c0], f1 = f[c1], f2 = f[c2], f3 = f[c3];
    if (f0 == parent) x += w0, ++c;
    if (f1 == parent) x += w1, ++c;
    if (f2 == parent) x += w2, ++c;
    if (f3 == parent) x += w3, ++c;
  }
  for (; p < b; p += step)
    if (f[col[p]] == parent) x += w[p], ++c;
}

__global__ void k_wsp_any(u32 n, const u64* off, const u32* col, const double* w, const u32* f,
                          const u32* s, const u8* cand, const u32* minmem, double* wsp,
                          unsigned long long* wcnt, u32* longrows, u32* nlong) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 v = warp; v < n; v += nwarps) {
    const u32 S = s[v];
    if (!cand[S]) continue;
    const u64 o0 = off[v], o1 = off[v + 1];
    if (o1 - o0 > LONG_ROW) {
      if (lane == 0) longrows[atomicAdd(nlong, 1u)] = (u32)v;
      continue;
    }
    const u32 parent = f[minmem[S]];
    double x = 0.0;
    unsigned long long c = 0;
    wsp_row_part(o0 + lane, o1, 32, col, w, f, parent, x, c);
    for (int o = 16; o; o >>= 1) {
      x += __shfl_xor_sync(0xffffffffu, x, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (lane == 0 && c) {
      atomicAdd(&wsp[S], x);
      atomicAdd(&wcnt[S], c);
    }
  }
}

__global__ void __launch_bounds__(256) k_wsp_any_long(const u32* longrows, const u32* nlong,
                                                      const u64* off, const u32* col,
                                                      const double* w, const u32* f, const u32* s,
                                                      const u32* minmem, double* wsp,
                                                      unsigned long long* wcnt) {
  __shared__ double sx[8];
  __shared__ unsigned long long sc[8];
  const u32 lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const u32 nl = *nlong;
  for (u32 t = blockIdx.x; t < nl; t += gridDim.x) {
    const u32 v = longrows[t];
    const u32 S = s[v];
    const u32 parent = f[minmem[S]];
    double x = 0.0;
    unsigned long long c = 0;
    wsp_row_part(off[v] + threadIdx.x, off[v + 1], 256, col, w, f, parent, x, c);
    for (int o = 16; o; o >>= 1) {
      x += __shfl_xor_sync(0xffffffffu, x, o);
      c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if (lane == 0) {
      sx[wib] = x;
      sc[wib] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double tx = 0.0;
      unsigned long long tc = 0;
      for (int j = 0; j < 8; ++j) tx += sx[j], tc += sc[j];
      if (tc) {
        atomicAdd(&wsp[S], tx);
        atomicAdd(&wcnt[S], tc);
      }
    }
    __syncthreads();
  }
}

// Ordered w(S, C_parent): members ascending, rows in CSR order, one chain per S
// (hit_leiden.rs:1618-1625).
__global__ void k_wsp_ordered(u32 nu, const u32* ukeys, const u32* ustart, u32 total,
                              const u32* members, const u64* off, const u32* col, const double* w,
                              const u32* f, const u32* minmem, double* wsp) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 j = warp; j < nu; j += nwarps) {
    u32 S = ukeys[j];
    u32 a = ustart[j], b = (j + 1 < nu) ? ustart[j + 1] : total;
    u32 parent = f[minmem[S]];
    double x = 0.0;
    for (u32 t = a; t < b; ++t) {
      u32 v = members[t];
      x = warp_ordered_sum(off[v], off[v + 1], x, [&](u64 p) { return w[p]; },
                           [&](u64 p) { return f[col[p]] == parent; });
    }
    if (lane == 0) wsp[S] = x;
  }
}

// T-filter decision from the any-order sum x of N positive terms.  The ordered
// sum the reference computes and x are both within γ_{N-1}·Σ of the exact sum
// (any summation tree of N terms), so they differ by at most
// 2γ_{N-1}/(1-γ_{N-1})·x < 2.0001·N·u·x (u = 2^-53); the window used here is
// 8·N·u·x, which also covers the rounding of the window itself.  ΔQ(S→∅) is
// non-increasing in w(S, C) (every rounding step is monotone), so the decision
// is certain when both ends of the window agree; otherwise S is flagged for
// the exact ordered sum.  With integral weights (exact in any order) or N <= 1
// the window is empty.
__global__ void k_blocked_bounds(u32 ns, const u8* cand, const double* dS, const double* wsp,
                                 const unsigned long long* wcnt, const u32* minmem,
                                 const u32* f, const double* dcomm, double tw, double gamma,
                                 bool exact_sums, bool force_exact, u8* blocked, u8* amb,
                                 u32* namb) {
  u32 local = 0;
  for (u64 S = blockIdx.x * (u64)blockDim.x + threadIdx.x; S < ns; S += (u64)gridDim.x * blockDim.x) {
    u8 b = 0, a = 0;
    if (cand[S]) {
      const double ds = dS[S];
      if (ds > 0.0) {
        const double dpar = dcomm[f[minmem[S]]];
        const double x = wsp[S];
        const unsigned long long N = wcnt[S];
        if (force_exact && N > 1) {
          a = 1;
        } else if (exact_sums || N <= 1) {
          b = remove_gain(x, tw, gamma, ds, dpar) > 1e-9 ? 1 : 0;
        } else {
          const double err = __dmul_rn(__dmul_rn(x, (double)N), 0x1p-50);
          const double lo = fmax(__dsub_rn(x, err), 0.0);
          const double hi = __dadd_rn(x, err);
          if (remove_gain(hi, tw, gamma, ds, dpar) > 1e-9) b = 1;
          else if (!(remove_gain(lo, tw, gamma, ds, dpar) > 1e-9)) b = 0;
          else a = 1;
        }
      }
    }
    blocked[S] = b;
    amb[S] = a;
    local += a;
  }
  if (local) atomicAdd(namb, local);
}

// Exact decision for the flagged S, from the ordered sum.
__global__ void k_blocked_exact(u32 ns, const u8* amb, const double* dS, const double* wsp,
                                const u32* minmem, const u32* f, const double* dcomm, double tw,
                                double gamma, u8* blocked) {
  for (u64 S = blockIdx.x * (u64)blockDim.x + threadIdx.x; S < ns; S += (u64)gridDim.x * blockDim.x) {
    if (!amb[S]) continue;
    const double dpar = dcomm[f[minmem[S]]];
    blocked[S] = remove_gain(wsp[S], tw, gamma, dS[S], dpar) > 1e-9 ? 1 : 0;
  }
}

__global__ void k_member_keys(u32 n, const u32* s, const u8* cand, u8* flag) {
  for (u64 v = blockIdx.x * (u64)blockDim.x + threadIdx.x; v < n; v += (u64)gridDim.x * blockDim.x)
    flag[v] = cand[s[v]] ? 1 : 0;
}

__global__ void k_gather_s(const u32* list, u32 m, const u32* s, u32* out) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < m; i += (u64)gridDim.x * blockDim.x)
    out[i] = s[list[i]];
}

__global__ void k_heads_u32b(const u32* sk, u64 n, u32* head) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    head[i] = (i == 0 || sk[i] != sk[i - 1]) ? 1u : 0u;
}

__global__ void k_seg_compact_b(const u32* head, const u32* segid, const u32* sk, u64 n,
                                u32* ukeys, u32* ustart) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    if (head[i]) {
      ukeys[segid[i]] = sk[i];
      ustart[segid[i]] = (u32)i;
    }
}

__global__ void k_apply_merges(const u32* single, u32 ns, const u32* to, const double* gain,
                               u32* s, u32* count) {
  u32 local = 0;
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < ns; i += (u64)gridDim.x * blockDim.x)
    if (gain[i] > 0.0) {
      s[single[i]] = to[i];
      ++local;
    }
  if (local) atomicAdd(count, local);
}

static u32 reduce_max_u32(Engine& E, const u32* x, u32 n, u32* out) {
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceReduce::Max(t, b, x, out, (int64_t)n, E.stream);
  });
  return E.read_u32(out);
}

static u32 select_flagged(Engine& E, const u8* flags, u32 n, u32* out, u32* cnt) {
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceSelect::Flagged(t, b, cub::CountingInputIterator<u32>(0), flags, out, cnt,
                                      (int64_t)n, E.stream);
  });
  return E.read_u32(cnt);
}

std::atomic<int> g_exact_tfilter{0};

RefineOut inc_refinement(Engine& E, Level& L, bool cc_same_community) {
  RefineOut out;
  Scratch& S = E.sc;
  cudaStream_t st = E.stream;
  const u32 n = L.g.n;
  E.new_ids.clear();
  S.refined.ensure(E.mem, n ? n : 1);
  HL_CUDA(cudaMemsetAsync(S.refined.p, 0, n ? n : 1, st));
  if (!n) return out;
  S.cnt.ensure(E.mem, 16);
  u32* cnt = S.cnt.p;
  u32* s = L.s_cur.p;

  // ---- 1. connected-component split of affected sub-communities ----------
  cudaEvent_t ev_cc = E.kt_begin();
  u32 smax = reduce_max_u32(E, s, n, cnt + 12);
  out.smax_before = smax;
  const size_t scap = (size_t)smax + 2 + n;
  S.affsc.ensure(E.mem, scap);
  HL_CUDA(cudaMemsetAsync(S.affsc.p, 0, scap, st));
  ++E.nlaunch, k_mark_affected_sc<<<grid_for(n), 256, 0, st>>>(S.affected.p, s, n, S.affsc.p);
  S.par.ensure(E.mem, n);
  S.csize.ensure(E.mem, n);
  ++E.nlaunch, k_iota<<<grid_for(n), 256, 0, st>>>(S.par.p, n);
  HL_CUDA(cudaMemsetAsync(S.csize.p, 0, sizeof(u32) * n, st));
  ++E.nlaunch, k_uf_edges<<<grid_for((u64)n * 32), 256, 0, st>>>(n, L.g.off.p, L.g.col.p, s, L.f.p, S.affsc.p,
                                                     cc_same_community, S.par.p);
  S.uroot.ensure(E.mem, n);
  ++E.nlaunch, k_uf_final<<<grid_for(n), 256, 0, st>>>(n, s, S.affsc.p, S.par.p, S.uroot.p,
                                                        S.csize.p);
  S.keep.ensure(E.mem, scap);
  HL_CUDA(cudaMemsetAsync(S.keep.p, 0, sizeof(u64) * scap, st));
  ++E.nlaunch, k_keep<<<grid_for(n), 256, 0, st>>>(n, s, S.affsc.p, S.uroot.p, S.csize.p,
                                      (unsigned long long*)S.keep.p);
  S.status.ensure(E.mem, n);
  S.gkey.ensure(E.mem, n);
  S.gkey2.ensure(E.mem, n);
  ++E.nlaunch, k_split_roots<<<grid_for(n), 256, 0, st>>>(n, s, S.affsc.p, S.uroot.p,
                                              (const unsigned long long*)S.keep.p, S.status.p,
                                              S.gkey.p);
  HL_LAUNCH_CHECK();
  S.act.ensure(E.mem, n);
  u32 m_new = select_flagged(E, S.status.p, n, S.act.p, cnt + 4);
  S.newid.ensure(E.mem, n);
  if (m_new) {
    S.keys.ensure(E.mem, m_new);
    S.keys2.ensure(E.mem, m_new);
    S.used.ensure(E.mem, m_new);
    S.rank.ensure(E.mem, m_new);
    ++E.nlaunch, k_gather_keys<<<grid_for(m_new), 256, 0, st>>>(S.act.p, m_new, S.gkey.p, S.keys.p);
    HL_LAUNCH_CHECK();
    u64* ki = S.keys.p;
    u64* ko = S.keys2.p;
    cub_run(E, [&](void* t, size_t& b) {
      return cub::DeviceRadixSort::SortKeys(t, b, ki, ko, (int64_t)m_new, 0, 64, st);
    });
    ++E.nlaunch, k_assign_newid<<<grid_for(m_new), 256, 0, st>>>(ko, m_new, smax + 1, S.newid.p, S.used.p,
                                                     S.rank.p);
    ++E.nlaunch, k_apply_split<<<grid_for(n), 256, 0, st>>>(n, s, S.affsc.p, S.uroot.p, S.status.p, S.newid.p,
                                               S.refined.p);
    HL_LAUNCH_CHECK();
    std::vector<u32> a(m_new), b(m_new);
    HL_CUDA(cudaMemcpyAsync(a.data(), S.used.p, sizeof(u32) * m_new, cudaMemcpyDeviceToHost, st));
    HL_CUDA(cudaMemcpyAsync(b.data(), S.rank.p, sizeof(u32) * m_new, cudaMemcpyDeviceToHost, st));
    E.sync();
    E.new_ids.resize(m_new);
    for (u32 i = 0; i < m_new; ++i) E.new_ids[i] = {a[i], b[i]};
  }
  out.splits = m_new;
  E.kt_end(KT_REFINE_CC, ev_cc);

  // is_initial (hit_leiden.rs:1333-1339): s is the identity ⇒ R = all
  // (decided on the device: no read-back).
  HL_CUDA(cudaMemsetAsync(cnt + 5, 0, sizeof(u32), st));
  ++E.nlaunch, k_not_identity<<<grid_for(n), 256, 0, st>>>(n, s, cnt + 5);
  ++E.nlaunch, k_refine_all_if_identity<<<grid_for(n), 256, 0, st>>>(n, cnt + 5, S.refined.p);
  HL_LAUNCH_CHECK();

  // ---- 2. sub-community sizes ------------------------------------------------
  u32 smax2 = m_new ? smax + m_new : smax;
  const size_t s2cap = (size_t)smax2 + 1;
  S.sizes.ensure(E.mem, s2cap);
  HL_CUDA(cudaMemsetAsync(S.sizes.p, 0, sizeof(u32) * s2cap, st));
  ++E.nlaunch, k_sizes<<<grid_for(n), 256, 0, st>>>(n, s, S.sizes.p);
  HL_LAUNCH_CHECK();

  // ---- 3. refined singletons ---------------------------------------------
  u32 nr = select_flagged(E, S.refined.p, n, S.act.p, cnt + 6);
  out.refined = nr;
  if (!nr) return out;
  if (E.cfg.mode == HL_MODE_DETERMINISTIC) {
    // sequential merges in (k, node) order with the live T-filter
    // (hit_leiden.rs:1392-1548)
    S.dS.ensure(E.mem, s2cap);
    recompute_comm_degrees(E, L, s, (u32)s2cap, S.dS.p);
    const size_t fcap = 2 * (size_t)n + 2;
    S.dcomm.ensure(E.mem, fcap);
    recompute_comm_degrees(E, L, L.f.p, (u32)fcap, S.dcomm.p);
    out.merges = merge_singletons_det(E, L, S.act.p, nr, S.sizes.p, S.dS.p, S.dcomm.p, s2cap);
    return out;
  }
  S.nmask.ensure(E.mem, nr);
  ++E.nlaunch, k_singletons<<<grid_for(nr), 256, 0, st>>>(S.act.p, nr, s, S.sizes.p, S.nmask.p);
  HL_LAUNCH_CHECK();
  S.cand_idx.ensure(E.mem, nr);
  u32 ns = 0;
  {
    u32* tmp = S.cand_idx.p;
    cub_run(E, [&](void* t, size_t& b) {
      return cub::DeviceSelect::Flagged(t, b, S.act.p, S.nmask.p, tmp, cnt + 7, (int64_t)nr, st);
    });
    ns = E.read_u32(cnt + 7);
  }
  if (!ns) return out;
  u32* single = S.cand_idx.p;
  // d_S and d_C serve only the T-filter and the singleton merges below
  S.dS.ensure(E.mem, s2cap);
  recompute_comm_degrees(E, L, s, (u32)s2cap, S.dS.p);
  const size_t fcap = 2 * (size_t)n + 2;
  S.dcomm.ensure(E.mem, fcap);
  recompute_comm_degrees(E, L, L.f.p, (u32)fcap, S.dcomm.p);

  // ---- 4. T-filter --------------------------------------------------------
  cudaEvent_t ev_tf = E.kt_begin();
  S.cand_sc.ensure(E.mem, s2cap);
  S.blocked.ensure(E.mem, s2cap);
  S.minmem.ensure(E.mem, s2cap);
  S.wsp.ensure(E.mem, s2cap);
  HL_CUDA(cudaMemsetAsync(S.cand_sc.p, 0, s2cap, st));
  HL_CUDA(cudaMemsetAsync(S.minmem.p, 0xFF, sizeof(u32) * s2cap, st));
  HL_CUDA(cudaMemsetAsync(S.wsp.p, 0, sizeof(double) * s2cap, st));
  S.wcnt.ensure(E.mem, s2cap);
  S.amb.ensure(E.mem, s2cap);
  HL_CUDA(cudaMemsetAsync(S.wcnt.p, 0, sizeof(u64) * s2cap, st));
  HL_CUDA(cudaMemsetAsync(cnt + 10, 0, 2 * sizeof(u32), st));
  ++E.nlaunch, k_t_candidates<<<grid_for((u64)ns * 32), 256, 0, st>>>(single, ns, L.g.off.p, L.g.col.p, L.f.p,
                                                         s, S.cand_sc.p);
  ++E.nlaunch, k_min_member<<<grid_for(n), 256, 0, st>>>(n, s, S.cand_sc.p, S.minmem.p);
  HL_LAUNCH_CHECK();
  // any-order w(S, C_parent) and term counts
  S.longrows.ensure(E.mem, n);
  unsigned long long* wcnt = reinterpret_cast<unsigned long long*>(S.wcnt.p);
  ++E.nlaunch, k_wsp_any<<<grid_for((u64)n * 32), 256, 0, st>>>(
      n, L.g.off.p, L.g.col.p, L.g.w.p, L.f.p, s, S.cand_sc.p, S.minmem.p, S.wsp.p, wcnt,
      S.longrows.p, cnt + 11);
  ++E.nlaunch, k_wsp_any_long<<<148 * 4, 256, 0, st>>>(S.longrows.p, cnt + 11, L.g.off.p, L.g.col.p,
                                                        L.g.w.p, L.f.p, s, S.minmem.p, S.wsp.p,
                                                        wcnt);
  ++E.nlaunch, k_blocked_bounds<<<grid_for(s2cap), 256, 0, st>>>(
      (u32)s2cap, S.cand_sc.p, S.dS.p, S.wsp.p, wcnt, S.minmem.p, L.f.p, S.dcomm.p, L.tw,
      E.cfg.resolution, E.integral, g_exact_tfilter.load() != 0, S.blocked.p, S.amb.p, cnt + 10);
  HL_LAUNCH_CHECK();
  const u32 namb = E.read_u32(cnt + 10);
  out.tfilter_exact = namb;
  if (namb) {
    // Ordered w(S, C_parent) for the undecided S: members sorted by (S, v).
    S.next.ensure(E.mem, n);
    ++E.nlaunch, k_member_keys<<<grid_for(n), 256, 0, st>>>(n, s, S.amb.p, S.next.p);
    HL_LAUNCH_CHECK();
    S.order.ensure(E.mem, n);
    u32 nm = select_flagged(E, S.next.p, n, S.order.p, cnt + 8);
    if (nm) {
      S.order2.ensure(E.mem, nm);
      S.used.ensure(E.mem, nm);
      S.rank.ensure(E.mem, nm);
      S.segid.ensure(E.mem, nm);
      S.rowlist.ensure(E.mem, nm);
      S.seg_start.ensure(E.mem, nm);
      S.sel_node.ensure(E.mem, nm);
      ++E.nlaunch, k_gather_s<<<grid_for(nm), 256, 0, st>>>(S.order.p, nm, s, S.used.p);
      HL_LAUNCH_CHECK();
      u32* ki = S.used.p;
      u32* ko = S.rank.p;
      u32* vi = S.order.p;
      u32* vo = S.order2.p;
      cub_run(E, [&](void* t, size_t& b) {
        return cub::DeviceRadixSort::SortPairs(t, b, ki, ko, vi, vo, (int64_t)nm, 0,
                                               bits_for(s2cap), st);
      });
      ++E.nlaunch, k_heads_u32b<<<grid_for(nm), 256, 0, st>>>(ko, nm, S.sel_node.p);
      HL_LAUNCH_CHECK();
      u32* h = S.sel_node.p;
      u32* sid = S.segid.p;
      cub_run(E, [&](void* t, size_t& b) {
        return cub::DeviceScan::ExclusiveSum(t, b, h, sid, (int64_t)nm, st);
      });
      u32 nu = E.read_u32(sid + nm - 1) + E.read_u32(h + nm - 1);
      ++E.nlaunch, k_seg_compact_b<<<grid_for(nm), 256, 0, st>>>(h, sid, ko, nm, S.rowlist.p, S.seg_start.p);
      ++E.nlaunch, k_wsp_ordered<<<grid_for((u64)nu * 32), 256, 0, st>>>(nu, S.rowlist.p, S.seg_start.p, nm, vo,
                                                  L.g.off.p, L.g.col.p, L.g.w.p, L.f.p,
                                                  S.minmem.p, S.wsp.p);
      HL_LAUNCH_CHECK();
    }
    ++E.nlaunch, k_blocked_exact<<<grid_for(s2cap), 256, 0, st>>>(
        (u32)s2cap, S.amb.p, S.dS.p, S.wsp.p, S.minmem.p, L.f.p, S.dcomm.p, L.tw,
        E.cfg.resolution, S.blocked.p);
    HL_LAUNCH_CHECK();
  }
  E.kt_end(KT_TFILTER, ev_tf);

  // ---- 5. Jacobi singleton merge -------------------------------------------
  S.cand_to.ensure(E.mem, ns);
  S.cand_gain.ensure(E.mem, ns);
  run_eval(E, 1, single, ns, L, s, S.dS.p, S.blocked.p, false, S.cand_to.p, S.cand_gain.p,
           nullptr);
  HL_CUDA(cudaMemsetAsync(cnt + 9, 0, sizeof(u32), st));
  ++E.nlaunch, k_apply_merges<<<grid_for(ns), 256, 0, st>>>(single, ns, S.cand_to.p, S.cand_gain.p, s,
                                               cnt + 9);
  HL_LAUNCH_CHECK();
  stats_acc_u32(E, cnt + 9, 9);  // merges, read when the call ends
  return out;
}

}  // namespace hl
