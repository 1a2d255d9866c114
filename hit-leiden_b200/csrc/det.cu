// det.cu — RunMode::Deterministic on the GPU: the sequential Gauss–Seidel
// movement (hit_leiden.rs:1103-1191) and the sequential singleton merges of
// the refinement (hit_leiden.rs:1392-1548).
//
// Both loops are sequential by definition: each step reads the state the
// previous step wrote.  They run as one persistent block that walks the
// vertices in the reference's order and spreads the work of each step (a
// row's neighbour scan, the candidate argmax, the frontier marks, a T-filter
// sum) over its threads, so a whole stage is one launch with no host round
// trip.  Results are bit-identical to the reference's steps under the
// canonical order used throughout (first CSR encounter for hash order):
//   * per-key sums are exact in any order with integral weights; with f64
//     weights one warp extends every key's sum in CSR order;
//   * strict '>' in first-encounter order = the largest gain, ties to the
//     smallest first CSR position;
//   * d(C), d_S and the sizes are updated in step order by one thread.
// No step waits on another block, and the loops are bounded (max_pops); a
// loop that reaches its bound stops and reports it through a status word.
#include <cstring>

#include "hl_engine.cuh"

namespace hl {

static inline u32 grid_for(u64 n, u32 block = 256) {
  u64 g = (n + block - 1) / block;
  if (g > 148u * 64u) g = 148u * 64u;
  return g ? (u32)g : 1u;
}

constexpr u32 DET_THREADS = 512;
constexpr u32 DET_WARPS = DET_THREADS / 32;
constexpr u32 DET_EMPTY = 0xFFFFFFFEu;  // "the next empty community" before an id is given

enum : u32 { DET_OK = 0, DET_POP_LIMIT = 1, DET_ID_SPACE = 2 };

// Σw and the first CSR position of every key of row [o0, o1) into the dense
// scratch (bw, bp), the distinct keys into klist (count in *nk).  `key(q)`
// returns the entry's key or NONE32 to skip it.  Integral weights: the whole
// block, atomics (every order gives the same sums).  Otherwise warp 0, in CSR
// order: a 32-entry tile at a time, entries of one key folded by its first
// lane in lane order, tiles in order.
template <typename K>
__device__ __forceinline__ void det_row_sums(u64 o0, u64 o1, const double* w, bool ordered,
                                             K key, double* bw, u32* bp, u32* klist, u32* nk,
                                             double* tile) {
  const u32 tid = threadIdx.x, lane = tid & 31;
  if (!ordered) {
    for (u64 q = o0 + tid; q < o1; q += DET_THREADS) {
      const u32 c = key(q);
      if (c == NONE32) continue;
      atomicAdd(&bw[c], w[q]);
      const u32 old = atomicMin(&bp[c], (u32)(q - o0));
      if (old == NONE32) klist[atomicAdd(nk, 1u)] = c;
    }
    return;
  }
  if (tid >= 32) return;
  for (u64 base = o0; base < o1; base += 32) {
    const u64 q = base + lane;
    const u32 c = q < o1 ? key(q) : NONE32;
    const bool ok = c != NONE32;
    tile[lane] = ok ? w[q] : 0.0;
    const u32 grp = __match_any_sync(0xffffffffu, ok ? (unsigned long long)c
                                                     : ((1ull << 32) | lane));
    __syncwarp();
    if (ok && lane == (u32)(__ffs(grp) - 1)) {
      if (bp[c] == NONE32) {
        bp[c] = (u32)(q - o0);
        klist[atomicAdd(nk, 1u)] = c;
      }
      double acc = bw[c];
      for (u32 m = grp; m; m &= m - 1) acc = __dadd_rn(acc, tile[__ffs(m) - 1]);
      bw[c] = acc;
    }
    __syncwarp();
  }
}

// Block argmax of (gain, first position, key) over positive gains: the
// largest gain, ties to the smallest position.  Returns in thread 0.
__device__ __forceinline__ void det_argmax(double& g, u32& p, u32& k, double* r_g, u32* r_p,
                                           u32* r_k) {
  const u32 tid = threadIdx.x, lane = tid & 31, wib = tid >> 5;
  for (int o = 16; o; o >>= 1) {
    const double og = __shfl_xor_sync(0xffffffffu, g, o);
    const u32 op = __shfl_xor_sync(0xffffffffu, p, o);
    const u32 ok = __shfl_xor_sync(0xffffffffu, k, o);
    if (op != NONE32 && (p == NONE32 || og > g || (og == g && op < p))) {
      g = og;
      p = op;
      k = ok;
    }
  }
  if (lane == 0) {
    r_g[wib] = g;
    r_p[wib] = p;
    r_k[wib] = k;
  }
  __syncthreads();
  if (tid == 0) {
    for (u32 x = 1; x < DET_WARPS; ++x) {
      if (r_p[x] != NONE32 && (p == NONE32 || r_g[x] > g || (r_g[x] == g && r_p[x] < p))) {
        g = r_g[x];
        p = r_p[x];
        k = r_k[x];
      }
    }
  }
}

struct DetMoveArgs {
  u32 n;
  const u64* off;
  const u32* col;
  const double* w;
  u32* f;
  const u32* s;
  const double* k;
  double* d;
  u64 dcap;            // entries of d (and of bw / bp): community ids stay below it
  u32* act;            // active bitset, (n + 31) / 32 words
  u8* changed;
  u8* affected;
  bool mark_moved;
  double* bw;          // dense per-community scratch: Σw (0.0 between rows)
  u32* bp;             // first CSR position (NONE32 between rows)
  u32* klist;          // the row's distinct keys
  double tw, gamma;
  u32 next_empty;      // id of the next empty community (hit_leiden.rs:1104)
  bool ordered;
  u64 max_pops;
  unsigned long long* out;  // [0] pops, [1] moves, [2] traversed, [3] status, [4] next_empty
};

// hit_leiden.rs:1103-1191.
__global__ void __launch_bounds__(DET_THREADS) k_det_move(DetMoveArgs A) {
  __shared__ u32 s_lo, s_found, s_nk, s_best, s_stop;
  __shared__ double s_bestg;
  __shared__ double r_g[DET_WARPS];
  __shared__ u32 r_p[DET_WARPS], r_k[DET_WARPS];
  __shared__ double tile[32];
  const u32 tid = threadIdx.x;
  const u32 nwords = (A.n + 31) >> 5;
  unsigned long long pops = 0, moves = 0, trav = 0;
  u32 next_empty = A.next_empty;
  if (tid == 0) {
    s_lo = 0;
    s_stop = DET_OK;
  }
  __syncthreads();
  while (true) {
    // 1. the lowest active vertex (iter_ones().next(), :1109)
    if (tid == 0) s_found = NONE32;
    __syncthreads();
    for (u32 base = s_lo; base < nwords; base += DET_THREADS) {
      const u32 wi = base + tid;
      const bool hit = wi < nwords && A.act[wi] != 0u;
      if (hit) atomicMin(&s_found, wi);
      if (__syncthreads_or(hit)) break;
    }
    const u32 word = s_found;
    if (word == NONE32) break;
    const u32 bits = A.act[word];
    const u32 v = (word << 5) + (u32)(__ffs(bits) - 1);
    __syncthreads();
    if (tid == 0) {
      A.act[word] = bits & (bits - 1u);
      s_lo = word;
      s_nk = 0;
      if (++pops > A.max_pops) s_stop = DET_POP_LIMIT;
    }
    __syncthreads();
    if (s_stop != DET_OK) break;
    const u64 o0 = A.off[v], o1 = A.off[v + 1];
    const u32 cur = A.f[v];
    const double kv = A.k[v];
    // 2. Σw per neighbour community, self-loops included (:1119-1125)
    const u32* f = A.f;
    const u32* col = A.col;
    det_row_sums(o0, o1, A.w, A.ordered, [&](u64 q) { return f[col[q]]; }, A.bw, A.bp, A.klist,
                 &s_nk, tile);
    __syncthreads();
    // 3. best candidate (:1127-1146), then the empty community (:1150-1162)
    const double wcur = A.bw[cur];
    const double dcur = A.d[cur];
    const u32 nk = s_nk;
    double g = 0.0;
    u32 p = NONE32, kk = NONE32;
    for (u32 i = tid; i < nk; i += DET_THREADS) {
      const u32 c = A.klist[i];
      if (c == cur) continue;
      const double gn = move_gain(A.bw[c], wcur, A.tw, A.gamma, kv, dcur, A.d[c]);
      const u32 pc = A.bp[c];
      if (gn > 0.0 && (p == NONE32 || gn > g || (gn == g && pc < p))) {
        g = gn;
        p = pc;
        kk = c;
      }
    }
    det_argmax(g, p, kk, r_g, r_p, r_k);
    if (tid == 0) {
      u32 best = cur;
      double bestg = 0.0;
      if (p != NONE32) {
        best = kk;
        bestg = g;
      }
      const double eg = empty_gain(wcur, A.tw, A.gamma, kv, dcur);
      if (eg > bestg) {
        bestg = eg;
        best = DET_EMPTY;
      }
      s_best = best;
      s_bestg = bestg;
      trav += o1 - o0;
    }
    __syncthreads();
    for (u32 i = tid; i < nk; i += DET_THREADS) {
      const u32 c = A.klist[i];
      A.bw[c] = 0.0;
      A.bp[c] = NONE32;
    }
    if (!(s_bestg > 0.0)) {  // :1164-1166
      __syncthreads();
      continue;
    }
    // 4. the move (:1168-1181)
    if (tid == 0) {
      u32 best = s_best;
      if (best == DET_EMPTY) {
        if ((u64)next_empty >= A.dcap) {
          s_stop = DET_ID_SPACE;
        } else {
          best = next_empty++;
        }
      }
      if (s_stop == DET_OK) {
        A.f[v] = best;
        A.changed[v] = 1;
        if (A.mark_moved) A.affected[v] = 1;
        A.d[cur] = __dsub_rn(A.d[cur], kv);
        A.d[best] = __dadd_rn(A.d[best], kv);
        s_best = best;
        ++moves;
      }
    }
    __syncthreads();
    if (s_stop != DET_OK) break;
    // 5. re-activate neighbours outside the new community, mark K (:1182-1187)
    const u32 best = s_best;
    const u32 sv = A.s[v];
    for (u64 q = o0 + tid; q < o1; q += DET_THREADS) {
      const u32 nb = A.col[q];
      if (A.f[nb] != best) {
        atomicOr(&A.act[nb >> 5], 1u << (nb & 31));
        atomicMin(&s_lo, nb >> 5);
      }
      if (A.s[nb] == sv) {
        A.affected[v] = 1;
        A.affected[nb] = 1;
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    A.out[0] = pops;
    A.out[1] = moves;
    A.out[2] = trav;
    A.out[3] = s_stop;
    A.out[4] = next_empty;
  }
}

__global__ void k_bits_from_flags(const u8* flags, u32 n, u32* bits) {
  const u32 nwords = (n + 31) >> 5;
  for (u64 wi = blockIdx.x * (u64)blockDim.x + threadIdx.x; wi < nwords;
       wi += (u64)gridDim.x * blockDim.x) {
    u32 x = 0;
    const u64 b = wi << 5;
    for (u32 j = 0; j < 32 && b + j < n; ++j)
      if (flags[b + j]) x |= 1u << j;
    bits[wi] = x;
  }
}

__global__ void k_fill_u32_det(u32* p, u32 v, u64 n) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    p[i] = v;
}

static void det_status(Engine& E, const u64* out, const char* stage) {
  if (out[3] == DET_POP_LIMIT)
    throw Error(HL_ERR_TIMEOUT, std::string(stage) + ": the sequential loop reached its step bound");
  if (out[3] == DET_ID_SPACE)
    throw Error(HL_ERR_UNSUPPORTED,
                std::string(stage) + ": more empty-community moves in one call than ids below 2n+2");
  (void)E;
}

// The deterministic branch of inc_movement, after seeding and d(C) (`active`
// holds A as 0/1 bytes).  Returns moves and traversed entries.
void inc_movement_det(Engine& E, Level& L, double* d, size_t dcap, bool mark_moved,
                      u64* moves, u64* traversed) {
  Scratch& S = E.sc;
  cudaStream_t st = E.stream;
  const u32 n = L.g.n;
  const u32 nwords = (n + 31) / 32;
  S.det_bits.ensure(E.mem, nwords ? nwords : 1);
  S.det_bw.ensure(E.mem, dcap);
  S.det_bp.ensure(E.mem, dcap);
  S.det_keys.ensure(E.mem, dcap);
  S.det_out.ensure(E.mem, 8);
  ++E.nlaunch, k_bits_from_flags<<<grid_for(nwords), 256, 0, st>>>(S.active.p, n, S.det_bits.p);
  HL_CUDA(cudaMemsetAsync(S.det_bw.p, 0, sizeof(double) * dcap, st));
  ++E.nlaunch, k_fill_u32_det<<<grid_for(dcap), 256, 0, st>>>(S.det_bp.p, NONE32, dcap);
  HL_CUDA(cudaMemsetAsync(S.det_out.p, 0, 8 * sizeof(u64), st));
  HL_LAUNCH_CHECK();
  DetMoveArgs A;
  A.n = n;
  A.off = L.g.off.p;
  A.col = L.g.col.p;
  A.w = L.g.w.p;
  A.f = L.f.p;
  A.s = L.s_cur.p;
  A.k = L.k.p;
  A.d = d;
  A.dcap = dcap;
  A.act = S.det_bits.p;
  A.changed = S.changed.p;
  A.affected = S.affected.p;
  A.mark_moved = mark_moved;
  A.bw = S.det_bw.p;
  A.bp = S.det_bp.p;
  A.klist = S.det_keys.p;
  A.tw = L.tw;
  A.gamma = E.cfg.resolution;
  A.next_empty = n;  // ids were compacted below n: the reference's community_degrees.len()
  A.ordered = !E.integral;
  A.max_pops = 4096ull * (u64)n + (1ull << 20);
  A.out = reinterpret_cast<unsigned long long*>(S.det_out.p);
  ++E.nlaunch, k_det_move<<<1, DET_THREADS, 0, st>>>(A);
  HL_LAUNCH_CHECK();
  u64 out[8];
  HL_CUDA(cudaMemcpyAsync(E.hs.p, S.det_out.p, 8 * sizeof(u64), cudaMemcpyDeviceToHost, st));
  E.sync();
  std::memcpy(out, E.hs.p, sizeof(out));
  det_status(E, out, "deterministic movement");
  *moves = out[1];
  *traversed = out[2];
}

// ----------------------------------------------------------------------------
// Sequential singleton merges with the live T-filter.
// ----------------------------------------------------------------------------
struct DetRefArgs {
  const u64* off;
  const u32* col;
  const double* w;
  const u32* f;
  u32* s;
  const double* k;
  double* dS;          // sub-community degrees (ordered sums, then step updates)
  u32* sizes;
  const double* dcomm; // d_parent: Σ k over each community, node order
  const u32* rlist;    // R sorted by (k, node)
  u32 nr;
  double* bw;
  u32* bp;
  u32* klist;
  double* wsp;         // cached w(S, C_parent)
  u8* wvalid;
  const u32* members;  // nodes sorted by (s, node) at the start of the merges
  const u32* mstart;   // per S: first index of its members (NONE32: none)
  const u32* mcount;   // per S: number of initial members
  u32* xhead;          // per S: merged singletons, ascending linked list
  u32* xnext;          // per node: next merged singleton of the same S
  double tw, gamma;
  bool ordered;
  unsigned long long* out;  // [0] merges
};

// w(S, C_parent) (hit_leiden.rs:1528-1541): S's members in node order (the
// initial ones and those merged since, two ascending lists), each member's
// row in CSR order, entries whose neighbour lies in C_parent.  With integral
// weights the block sums in any order; otherwise warp 0 folds in that order.
__device__ double det_wsp(const DetRefArgs& A, u32 S, u32 parent, double* r_g) {
  const u32 tid = threadIdx.x, lane = tid & 31, wib = tid >> 5;
  const u32 ms = A.mstart[S];
  const u32 mc = ms == NONE32 ? 0u : A.mcount[S];
  const u32* f = A.f;
  const u32* col = A.col;
  const double* w = A.w;
  if (!A.ordered) {
    double acc = 0.0;
    // initial members: a warp per member row
    for (u32 i = wib; i < mc; i += DET_WARPS) {
      const u32 m = A.members[ms + i];
      for (u64 q = A.off[m] + lane; q < A.off[m + 1]; q += 32)
        if (f[col[q]] == parent) acc += w[q];
    }
    // merged singletons
    for (u32 m = A.xhead[S]; m != NONE32; m = A.xnext[m])
      for (u64 q = A.off[m] + tid; q < A.off[m + 1]; q += DET_THREADS)
        if (f[col[q]] == parent) acc += w[q];
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) r_g[wib] = acc;
    __syncthreads();
    double tot = 0.0;
    if (tid == 0)
      for (u32 x = 0; x < DET_WARPS; ++x) tot += r_g[x];
    __syncthreads();
    return tot;  // thread 0
  }
  double acc = 0.0;
  if (tid < 32) {
    u32 i = 0;
    u32 x = A.xhead[S];
    while (i < mc || x != NONE32) {
      u32 m;
      if (x == NONE32 || (i < mc && A.members[ms + i] < x)) {
        m = A.members[ms + i];
        ++i;
      } else {
        m = x;
        x = A.xnext[x];
      }
      acc = warp_ordered_sum(A.off[m], A.off[m + 1], acc, [&](u64 t) { return w[t]; },
                             [&](u64 t) { return f[col[t]] == parent; });
    }
  }
  __syncthreads();
  return acc;  // thread 0 (all of warp 0)
}

// hit_leiden.rs:1392-1413 → try_merge_singleton_refinement (:1419-1511) with
// should_skip_candidate_t_filter (:1514-1548).
__global__ void __launch_bounds__(DET_THREADS) k_det_refine(DetRefArgs A) {
  __shared__ u32 s_nk, s_best, s_v, s_go;
  __shared__ double s_bestg, s_wsp;
  __shared__ double r_g[DET_WARPS];
  __shared__ u32 r_p[DET_WARPS], r_k[DET_WARPS];
  __shared__ double tile[32];
  const u32 tid = threadIdx.x;
  unsigned long long merges = 0;
  for (u32 i = 0; i < A.nr; ++i) {
    const u32 v = A.rlist[i];
    const u32 cs = A.s[v];
    if (A.sizes[cs] != 1u) continue;  // singleton check (:1398-1400), uniform
    const u32 cc = A.f[v];
    const double kv = A.k[v];
    if (tid == 0) s_nk = 0;
    __syncthreads();
    const u32* f = A.f;
    const u32* col = A.col;
    const u32* s = A.s;
    det_row_sums(A.off[v], A.off[v + 1], A.w, A.ordered,
                 [&](u64 q) {
                   const u32 nb = col[q];
                   return f[nb] == cc ? s[nb] : NONE32;
                 },
                 A.bw, A.bp, A.klist, &s_nk, tile);
    __syncthreads();
    const double wcur = A.bw[cs];
    const double dcs = A.dS[cs];
    const double dpar = A.dcomm[cc];
    const u32 nk = s_nk;
    // Candidates in gain order; the best one the T-filter lets through wins
    // (the same choice as the reference's strict '>' over the filtered list).
    if (tid == 0) {
      s_best = cs;
      s_bestg = 0.0;
      s_go = 1;
    }
    __syncthreads();
    while (s_go) {
      double g = 0.0;
      u32 p = NONE32, kk = NONE32;
      for (u32 j = tid; j < nk; j += DET_THREADS) {
        const u32 c = A.klist[j];
        if (c == cs || A.bp[c] == NONE32 - 1u) continue;  // current, or filtered out
        const double gn = move_gain(A.bw[c], wcur, A.tw, A.gamma, kv, dcs, A.dS[c]);
        const u32 pc = A.bp[c];
        if (gn > 0.0 && (p == NONE32 || gn > g || (gn == g && pc < p))) {
          g = gn;
          p = pc;
          kk = c;
        }
      }
      det_argmax(g, p, kk, r_g, r_p, r_k);
      if (tid == 0) {
        s_v = p == NONE32 ? NONE32 : kk;
        s_bestg = g;
      }
      __syncthreads();
      const u32 cand = s_v;
      if (cand == NONE32) {
        if (tid == 0) s_go = 0;
        __syncthreads();
        break;
      }
      // T-filter of the candidate (:1514-1548)
      const double ds = A.dS[cand];
      bool skip = false;
      if (ds > 0.0) {
        double x;
        if (A.wvalid[cand]) {
          x = A.wsp[cand];
        } else {
          x = det_wsp(A, cand, cc, r_g);
          if (tid == 0) {
            A.wsp[cand] = x;
            A.wvalid[cand] = 1;
          }
        }
        if (tid == 0) s_wsp = x;
        __syncthreads();
        skip = remove_gain(s_wsp, A.tw, A.gamma, ds, dpar) > 1e-9;
      }
      if (tid == 0) {
        if (skip) {
          A.bp[cand] = NONE32 - 1u;  // filtered out for this vertex
        } else {
          s_best = cand;
          s_go = 0;
        }
      }
      __syncthreads();
    }
    const u32 best = s_best;
    const double bestg = s_bestg;
    // the row's same-community weight, for the merged vertex's T-filter share
    __syncthreads();
    for (u32 j = tid; j < nk; j += DET_THREADS) {
      const u32 c = A.klist[j];
      A.bw[c] = 0.0;
      A.bp[c] = NONE32;
    }
    __syncthreads();
    if (best != cs && bestg > 0.0) {
      if (tid == 0) {
        A.s[v] = best;
        A.sizes[cs] -= 1u;
        A.sizes[best] += 1u;
        A.dS[cs] = __dsub_rn(A.dS[cs], kv);
        A.dS[best] = __dadd_rn(A.dS[best], kv);
        ++merges;
        // v joins best's members, in node order
        u32* link = &A.xhead[best];
        while (*link != NONE32 && *link < v) link = &A.xnext[*link];
        A.xnext[v] = *link;
        *link = v;
        A.wvalid[best] = 0;  // w(best, C) is summed again when next needed
      }
      __syncthreads();
    }
  }
  if (tid == 0) A.out[0] = merges;
}

__global__ void k_member_index(const u32* sorted_s, u32 n, u32* mstart, u32* mcount) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
    const u32 c = sorted_s[i];
    if (i == 0 || sorted_s[i - 1] != c) mstart[c] = (u32)i;
    atomicAdd(&mcount[c], 1u);
  }
}

__global__ void k_k_keys(const u32* verts, u32 nv, const double* k, u64* keys) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < nv; i += (u64)gridDim.x * blockDim.x)
    keys[i] = double_key(k[verts[i]]);
}

__global__ void k_iota_det(u32* p, u32 n) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    p[i] = (u32)i;
}

// The deterministic merge step of inc_refinement: refined vertices `rv`
// (ascending, nr of them), sub-community sizes and degrees for ids < scap,
// d_parent per community.  Returns the number of merges.
u64 merge_singletons_det(Engine& E, Level& L, const u32* rv, u32 nr, u32* sizes, double* dS,
                         const double* dcomm, size_t scap) {
  Scratch& S = E.sc;
  cudaStream_t st = E.stream;
  const u32 n = L.g.n;
  u32* s = L.s_cur.p;
  // R sorted by k ascending, stable (hit_leiden.rs:1373-1374)
  S.det_k64.ensure(E.mem, nr);
  S.det_k64b.ensure(E.mem, nr);
  S.det_rsort.ensure(E.mem, nr);
  ++E.nlaunch, k_k_keys<<<grid_for(nr), 256, 0, st>>>(rv, nr, L.k.p, S.det_k64.p);
  HL_LAUNCH_CHECK();
  {
    u64* ki = S.det_k64.p;
    u64* ko = S.det_k64b.p;
    const u32* vi = rv;
    u32* vo = S.det_rsort.p;
    cub_run(E, [&](void* t, size_t& b) {
      return cub::DeviceRadixSort::SortPairs(t, b, ki, ko, vi, vo, (int64_t)nr, 0, 64, st);
    });
  }
  // nodes by (s, node): the initial members of every sub-community
  S.det_mkey.ensure(E.mem, n);
  S.det_mkey2.ensure(E.mem, n);
  S.det_mval.ensure(E.mem, n);
  S.det_members.ensure(E.mem, n);
  S.det_mstart.ensure(E.mem, scap);
  S.det_mcount.ensure(E.mem, scap);
  S.det_xhead.ensure(E.mem, scap);
  S.det_xnext.ensure(E.mem, n);
  S.det_wsp.ensure(E.mem, scap);
  S.det_wvalid.ensure(E.mem, scap);
  S.det_bw.ensure(E.mem, scap);
  S.det_bp.ensure(E.mem, scap);
  S.det_keys.ensure(E.mem, scap);
  S.det_out.ensure(E.mem, 8);
  HL_CUDA(cudaMemcpyAsync(S.det_mkey.p, s, sizeof(u32) * n, cudaMemcpyDeviceToDevice, st));
  ++E.nlaunch, k_iota_det<<<grid_for(n), 256, 0, st>>>(S.det_mval.p, n);
  HL_LAUNCH_CHECK();
  {
    u32* ki = S.det_mkey.p;
    u32* ko = S.det_mkey2.p;
    u32* vi = S.det_mval.p;
    u32* vo = S.det_members.p;
    cub_run(E, [&](void* t, size_t& b) {
      return cub::DeviceRadixSort::SortPairs(t, b, ki, ko, vi, vo, (int64_t)n, 0,
                                             bits_for(scap), st);
    });
  }
  ++E.nlaunch, k_fill_u32_det<<<grid_for(scap), 256, 0, st>>>(S.det_mstart.p, NONE32, scap);
  HL_CUDA(cudaMemsetAsync(S.det_mcount.p, 0, sizeof(u32) * scap, st));
  ++E.nlaunch, k_member_index<<<grid_for(n), 256, 0, st>>>(S.det_mkey2.p, n, S.det_mstart.p,
                                                            S.det_mcount.p);
  ++E.nlaunch, k_fill_u32_det<<<grid_for(scap), 256, 0, st>>>(S.det_xhead.p, NONE32, scap);
  ++E.nlaunch, k_fill_u32_det<<<grid_for(scap), 256, 0, st>>>(S.det_bp.p, NONE32, scap);
  HL_CUDA(cudaMemsetAsync(S.det_wvalid.p, 0, scap, st));
  HL_CUDA(cudaMemsetAsync(S.det_bw.p, 0, sizeof(double) * scap, st));
  HL_CUDA(cudaMemsetAsync(S.det_out.p, 0, 8 * sizeof(u64), st));
  HL_LAUNCH_CHECK();
  DetRefArgs A;
  A.off = L.g.off.p;
  A.col = L.g.col.p;
  A.w = L.g.w.p;
  A.f = L.f.p;
  A.s = s;
  A.k = L.k.p;
  A.dS = dS;
  A.sizes = sizes;
  A.dcomm = dcomm;
  A.rlist = S.det_rsort.p;
  A.nr = nr;
  A.bw = S.det_bw.p;
  A.bp = S.det_bp.p;
  A.klist = S.det_keys.p;
  A.wsp = S.det_wsp.p;
  A.wvalid = S.det_wvalid.p;
  A.members = S.det_members.p;
  A.mstart = S.det_mstart.p;
  A.mcount = S.det_mcount.p;
  A.xhead = S.det_xhead.p;
  A.xnext = S.det_xnext.p;
  A.tw = L.tw;
  A.gamma = E.cfg.resolution;
  A.ordered = !E.integral;
  A.out = reinterpret_cast<unsigned long long*>(S.det_out.p);
  ++E.nlaunch, k_det_refine<<<1, DET_THREADS, 0, st>>>(A);
  HL_LAUNCH_CHECK();
  return E.read_u64(S.det_out.p);
}

}  // namespace hl
