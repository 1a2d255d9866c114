// eval.cu — best-move evaluation on a fixed snapshot, shared by inc-movement
// (parallel_frontier.rs:133-239) and the refinement merge
// (throughput.rs:291-359).
//
// For every listed vertex v: Σw(v, X) per neighbour key X (community for the
// movement, sub-community inside v's community for the refinement), each sum
// extended in CSR order; then the argmax of the FP64 gain with the reference's
// tie rule (strict '>' in first-encounter order = on equal gains the smallest
// first CSR position); then, for the movement, the empty community n+v on a
// strict improvement.
//
// Vertices are binned by degree so that no lane idles on short rows and no
// vertex waits on a table far larger than it needs:
//   deg <= 8, 16, 32    sub-warp groups of 8 / 16 / 32 lanes, one chunk, no table;
//   33 .. MID_MAX       a warp per vertex, shared-memory table sized 2·deg;
//   MID_MAX .. WIDE_MAX a warp per vertex, a per-warp shared-memory table
//                       (half-size tables up to WIDE_SPLIT);
//   larger              a block per vertex: 256-entry adjacency tiles bucketed
//                       by a hash partition of their keys, one partition per
//                       warp, each warp folding its own keys in CSR order into
//                       a shared table of 4096 slots (a second pass with
//                       global tables takes rows with more than 2048 distinct
//                       keys), so every key's sum keeps the reference's
//                       rounding.
#include <cstring>

#include "hl_engine.cuh"

namespace hl {

static inline u32 grid_for(u64 n, u32 block = 256) {
  u64 g = (n + block - 1) / block;
  if (g > 148u * 64u) g = 148u * 64u;
  return g ? (u32)g : 1u;
}

enum EvalKind { EVAL_MOVE = 0, EVAL_REFINE = 1 };

struct EvalArgs {
  const u32* verts;   // vertex ids
  const u32* idx;     // indices into verts handled by this launch
  u32 nidx;
  const u64* off;
  const u32* col;
  const double* w;
  const u32* f;
  const u32* s;
  const double* d;
  const double* kdeg;
  const u8* blocked;
  double tw, gamma;
  u32 n;
  bool allow_empty;
  bool concurrent;  // integral weights: order-free accumulation allowed
  u32* out_to;
  double* out_gain;
  u32* tkey;
  u32* tpos;
  double* tval;
  u32* tlist;    // per-warp / per-block insertion lists of used slots
  u64 region;    // table entries per block region (block kernel)
  unsigned long long* counters;  // [0] entries scanned, [1] candidates evaluated
  u32* ovf_list;   // block kernel without global regions: rows deferred because
  u32* ovf_count;  // they passed BIG_TAB / 2 distinct keys (idx values)
  const u32* nidx_dev;  // if set, the number of idx entries is read here
  u32* work;            // block kernel: next idx position to take (zeroed per launch)
  u64 defer_deg;        // block kernel pass 1: rows longer than this go to the
                        // partitioned pass unread (0: none)
};

constexpr u32 MID_MAX = 128;
constexpr u32 MID_TAB = 256;  // per-warp table entries (>= 2 * MID_MAX)
constexpr u32 MID_WARPS = 8;
constexpr u32 BIG_THREADS = 256;


__device__ __forceinline__ u32 hash32(u32 x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// Integral weights and sums in [0, 2^52) (the handle keeps 2m below 2^52, and
// every partial sum of a row is at most its k_v) between double and integer
// without a conversion instruction: 2^52 + x is exact there, and its bits are
// those of 2^52 plus x.
constexpr double TWO52 = 4503599627370496.0;
constexpr unsigned long long TWO52_BITS = 0x4330000000000000ull;
__device__ __forceinline__ unsigned long long int_of(double w) {
  return (unsigned long long)__double_as_longlong(__dadd_rn(w, TWO52)) - TWO52_BITS;
}
__device__ __forceinline__ double dbl_of(unsigned long long s) {
  return __dsub_rn(__longlong_as_double((long long)(s + TWO52_BITS)), TWO52);
}

// Sum and smallest position of each match_any group of a warp (grp: this
// lane's group; w < 2^26 on every lane, so a group's sum fits 32 bits).  A
// lane alone in its group keeps its own values.  The groups of two or more
// lanes (in a chunk of a hub row these are its few heavy keys) take one
// full-warp reduction each: reductions whose lanes name different masks
// would run once per distinct mask, which a chunk of mostly distinct keys
// turns into 32.
__device__ __forceinline__ void group_sums(u32 grp, u32 lane, bool valid, u32 w, u32 pos,
                                           unsigned long long& sum, u32& pmin) {
  sum = w;
  pmin = pos;
  u32 multi = __ballot_sync(0xffffffffu, valid && (grp & (grp - 1)) != 0 &&
                                              lane == (u32)(__ffs(grp) - 1));
  while (multi) {
    const u32 l = __ffs(multi) - 1;
    const u32 gm = __shfl_sync(0xffffffffu, grp, l);
    const bool in = (gm >> lane) & 1u;
    const u32 s = __reduce_add_sync(0xffffffffu, in ? w : 0u);
    const u32 m = __reduce_min_sync(0xffffffffu, in ? pos : 0xFFFFFFFFu);
    if (lane == l) {
      sum = s;
      pmin = m;
    }
    multi &= multi - 1;
  }
}

template <int KIND>
__device__ __forceinline__ bool entry_key(const EvalArgs& A, u32 v, u32 nb, u32 fv, u32& key) {
  if (KIND == EVAL_MOVE) {
    if (nb == v) return false;  // self-loops skipped (parallel_frontier.rs:164-166)
    key = A.f[nb];
    return true;
  } else {
    if (A.f[nb] != fv) return false;  // same community only (throughput.rs:308-311)
    key = A.s[nb];
    return true;
  }
}

// Final decision of one vertex from its best neighbour candidate.
template <int KIND>
__device__ __forceinline__ void finish(const EvalArgs& A, u32 i, u32 v, u32 cur, double kv,
                                       double wcur, double best_g, u32 best_key, bool has_best) {
  u32 to = cur;
  double g = 0.0;
  if (has_best && best_g > 0.0) {
    g = best_g;
    to = best_key;
  }
  if (KIND == EVAL_MOVE && A.allow_empty && A.tw != 0.0) {
    double eg = empty_gain(wcur, A.tw, A.gamma, kv, A.d[cur]);
    if (eg > g) {
      g = eg;
      to = A.n + v;
    }
  }
  A.out_to[i] = to;
  A.out_gain[i] = g;
}

__device__ __forceinline__ void block_count(const EvalArgs& A, unsigned long long trav,
                                            unsigned long long cand) {
  if (!A.counters) return;
  for (int o = 16; o; o >>= 1) {
    trav += __shfl_xor_sync(0xffffffffu, trav, o);
    cand += __shfl_xor_sync(0xffffffffu, cand, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (trav) atomicAdd(&A.counters[0], trav);
    if (cand) atomicAdd(&A.counters[1], cand);
  }
}

// ---------------------------------------------------------------------------
// Small degrees: groups of G lanes, one vertex per group, one chunk.
// ---------------------------------------------------------------------------
template <int KIND, int G>
__global__ void __launch_bounds__(256) k_eval_small(EvalArgs A) {
  __shared__ double s_w[256];
  const u32 lane = threadIdx.x & 31;
  const u32 grp_in_warp = lane / G;
  const u32 gl = lane % G;
  const u32 gbase = lane - gl;  // first lane of this group
  const u32 gmask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << gbase);
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  constexpr u32 GPW = 32 / G;
  unsigned long long trav = 0, ncand = 0;
  for (u64 base = warp * GPW; base < A.nidx; base += nwarps * GPW) {
    const u64 t = base + grp_in_warp;
    const bool live = t < A.nidx;
    u32 i = 0, v = 0, cur = 0, fv = 0;
    u64 o0 = 0, deg = 0;
    double kv = 0.0;
    if (live) {
      i = A.idx[t];
      v = A.verts[i];
      o0 = A.off[v];
      deg = A.off[v + 1] - o0;
      fv = A.f[v];
      cur = (KIND == EVAL_MOVE) ? fv : A.s[v];
      kv = A.kdeg[v];
      if (gl == 0) trav += deg;
    }
    u32 key = NONE32;
    double wv = 0.0;
    bool has = false;
    if (live && gl < deg) {
      u32 nb = A.col[o0 + gl];
      wv = A.w[o0 + gl];
      has = entry_key<KIND>(A, v, nb, fv, key);
    }
    s_w[threadIdx.x] = wv;
    __syncwarp();
    unsigned long long mv = has ? (((unsigned long long)grp_in_warp << 32) | key)
                                : (0x8000000000000000ull | lane);
    u32 grp = __match_any_sync(0xffffffffu, mv);
    bool leader = has && lane == (u32)(__ffs(grp) - 1);
    double sum = 0.0;
    if (leader)
      for (u32 m = grp; m; m &= m - 1)
        sum = __dadd_rn(sum, s_w[(threadIdx.x & ~31u) + __ffs(m) - 1]);
    u32 curm = __ballot_sync(0xffffffffu, leader && key == cur) & gmask;
    double wc = __shfl_sync(0xffffffffu, sum, curm ? (__ffs(curm) - 1) : lane);
    double wcur = curm ? wc : 0.0;
    double g = -1.0;
    u32 p = NONE32, kk = key;
    if (leader && key != cur && A.tw != 0.0) {
      bool blk = (KIND == EVAL_REFINE) && A.blocked[key];
      if (!blk) {
        g = move_gain(sum, wcur, A.tw, A.gamma, kv, A.d[cur], A.d[key]);
        p = gl;
        ++ncand;
      }
    }
#pragma unroll
    for (int o = G / 2; o; o >>= 1) {
      double og = __shfl_xor_sync(0xffffffffu, g, o);
      u32 op = __shfl_xor_sync(0xffffffffu, p, o);
      u32 ok = __shfl_xor_sync(0xffffffffu, kk, o);
      if (op != NONE32 && (p == NONE32 || og > g || (og == g && op < p))) {
        g = og;
        p = op;
        kk = ok;
      }
    }
    if (live && gl == 0) finish<KIND>(A, i, v, cur, kv, wcur, g, kk, p != NONE32);
    __syncwarp();
  }
  block_count(A, trav, ncand);
}

// ---------------------------------------------------------------------------
// Mid degrees: a warp per vertex with a shared table sized to the vertex.
// The row's chunks (at most MID_MAX / 32) are loaded together and their keys
// gathered together, then folded in CSR order; the candidates' community
// degrees are gathered MID_SCAN_UNROLL at a time.
// ---------------------------------------------------------------------------
constexpr u32 MID_CHUNKS = MID_MAX / 32;
constexpr u32 MID_SCAN_UNROLL = 4;

template <int KIND>
__global__ void __launch_bounds__(MID_WARPS * 32, 4) k_eval_mid(EvalArgs A) {
  __shared__ u32 s_key[MID_WARPS][MID_TAB];
  __shared__ u32 s_pos[MID_WARPS][MID_TAB];
  __shared__ double s_val[MID_WARPS][MID_TAB];
  __shared__ double s_w[MID_WARPS][MID_CHUNKS * 32];
  const u32 lane = threadIdx.x & 31;
  const u32 wib = threadIdx.x >> 5;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  unsigned long long trav = 0, ncand = 0;
  u32* tk = s_key[wib];
  u32* tp = s_pos[wib];
  double* tv = s_val[wib];
  double* sw = s_w[wib];
  // the next vertex's list entry, id and row bounds, one step at a time
  u32 i_nx = 0, v_nx = 0;
  u64 o0_nx = 0, o1_nx = 0;
  if (warp < A.nidx) {
    i_nx = A.idx[warp];
    v_nx = A.verts[i_nx];
    o0_nx = A.off[v_nx];
    o1_nx = A.off[v_nx + 1];
  }
  for (u64 t = warp; t < A.nidx; t += nwarps) {
    const u32 i = i_nx;
    const u32 v = v_nx;
    const u64 o0 = o0_nx, o1 = o1_nx;
    const u64 deg = o1 - o0;
    const bool has_nx = t + nwarps < A.nidx;
    if (has_nx) i_nx = A.idx[t + nwarps];
    const u32 fv = A.f[v];
    const u32 cur = (KIND == EVAL_MOVE) ? fv : A.s[v];
    const double kv = A.kdeg[v];
    const double dcur = A.d[cur];
    if (lane == 0) trav += deg;
    u32 cap = 64;
    while (cap < 2 * deg) cap <<= 1;
    const u32 mask = cap - 1;
    for (u32 x = lane; x < cap; x += 32) tk[x] = NONE32;
    u32 nb[MID_CHUNKS], key[MID_CHUNKS];
#pragma unroll
    for (u32 j = 0; j < MID_CHUNKS; ++j) {
      const u64 q = o0 + j * 32 + lane;
      nb[j] = NONE32;
      double wv = 0.0;
      if (q < o1) {
        nb[j] = A.col[q];
        wv = A.w[q];
      }
      sw[j * 32 + lane] = wv;
    }
#pragma unroll
    for (u32 j = 0; j < MID_CHUNKS; ++j) {
      key[j] = NONE32;
      if (nb[j] != NONE32 && !entry_key<KIND>(A, v, nb[j], fv, key[j])) key[j] = NONE32;
    }
    if (has_nx) v_nx = A.verts[i_nx];
    __syncwarp();
#pragma unroll
    for (u32 j = 0; j < MID_CHUNKS; ++j) {
      if (o0 + j * 32 >= o1) break;  // warp-uniform
      const u64 q = o0 + j * 32 + lane;
      const u32 grp = __match_any_sync(0xffffffffu, key[j]);
      if (key[j] != NONE32 && lane == (u32)(__ffs(grp) - 1)) {
        u32 slot = hash32(key[j]) & mask;
        while (true) {
          u32 prev = atomicCAS(&tk[slot], NONE32, key[j]);
          if (prev == NONE32 || prev == key[j]) {
            double sum = prev == NONE32 ? 0.0 : tv[slot];
            for (u32 m = grp; m; m &= m - 1) sum = __dadd_rn(sum, sw[j * 32 + __ffs(m) - 1]);
            tv[slot] = sum;
            if (prev == NONE32) tp[slot] = (u32)(q - o0);
            break;
          }
          slot = (slot + 1) & mask;
        }
      }
      __syncwarp();
    }
    double wcur = 0.0;
    bool found = false;
    for (u32 x = lane; x < cap; x += 32)
      if (tk[x] == cur) {
        wcur = tv[x];
        found = true;
      }
    u32 fm = __ballot_sync(0xffffffffu, found);
    wcur = __shfl_sync(0xffffffffu, wcur, fm ? __ffs(fm) - 1 : 0);
    if (!fm) wcur = 0.0;
    if (has_nx) {
      o0_nx = A.off[v_nx];
      o1_nx = A.off[v_nx + 1];
    }
    double g = -1.0;
    u32 p = NONE32, kk = cur;
    if (A.tw != 0.0) {
      GainScreen scr;  // exact gains only for candidates that may win
      scr.init(wcur, A.tw, A.gamma, kv, dcur);
      for (u32 x0 = lane; x0 < cap; x0 += 32 * MID_SCAN_UNROLL) {
        u32 kq[MID_SCAN_UNROLL];
        double dk[MID_SCAN_UNROLL];
#pragma unroll
        for (u32 j = 0; j < MID_SCAN_UNROLL; ++j) {
          const u32 x = x0 + 32 * j;
          kq[j] = x < cap ? tk[x] : NONE32;
          if (kq[j] == cur) kq[j] = NONE32;
          if (KIND == EVAL_REFINE && kq[j] != NONE32 && A.blocked[kq[j]]) kq[j] = NONE32;
        }
#pragma unroll
        for (u32 j = 0; j < MID_SCAN_UNROLL; ++j) dk[j] = kq[j] != NONE32 ? A.d[kq[j]] : 0.0;
#pragma unroll
        for (u32 j = 0; j < MID_SCAN_UNROLL; ++j) {
          if (kq[j] == NONE32) continue;
          const u32 x = x0 + 32 * j;
          ++ncand;
          if (!scr.keep(tv[x], dk[j])) continue;
          const double gn = move_gain(tv[x], wcur, A.tw, A.gamma, kv, dcur, dk[j]);
          const u32 pp = tp[x];
          if (p == NONE32 || gn > g || (gn == g && pp < p)) {
            g = gn;
            p = pp;
            kk = kq[j];
          }
        }
      }
    }
    for (int o = 16; o; o >>= 1) {
      double og = __shfl_xor_sync(0xffffffffu, g, o);
      u32 op = __shfl_xor_sync(0xffffffffu, p, o);
      u32 ok = __shfl_xor_sync(0xffffffffu, kk, o);
      if (op != NONE32 && (p == NONE32 || og > g || (og == g && op < p))) {
        g = og;
        p = op;
        kk = ok;
      }
    }
    if (lane == 0) finish<KIND>(A, i, v, cur, kv, wcur, g, kk, p != NONE32);
    __syncwarp();
  }
  block_count(A, trav, ncand);
}

// ---------------------------------------------------------------------------
// Wide degrees (MID_MAX < deg <= WIDE_MAX): a warp per vertex.  The warp
// issues the loads of up to 8 chunks (256 entries) at once, then folds the
// chunks in CSR order into its own shared-memory table (TAB = 2 x the bin's
// largest degree slots: keys, 16-bit first positions, sums).  Every new key's
// slot is appended to a per-warp list, so the argmax scan visits only used
// slots and resets them: the table is clean again for the warp's next vertex
// without a clearing pass.  The bin is split at WIDE_SPLIT: rows up to it
// take half-size tables, so more warps fit on an SM.
// ---------------------------------------------------------------------------
constexpr u32 WIDE_MAX = 512;
constexpr u32 WIDE_SPLIT = 256;
constexpr u32 WIDE_WARPS = 4;
constexpr u32 WIDE_BATCH = 8;  // chunks loaded before folding
constexpr u32 WIDE_SCAN_UNROLL = 4;  // table slots whose community degrees are gathered together

template <u32 TAB>
struct WideSmem {
  double tv[WIDE_WARPS][TAB];
  double sw[WIDE_WARPS][WIDE_BATCH * 32];
  u32 tk[WIDE_WARPS][TAB];
  unsigned short tp[WIDE_WARPS][TAB];
  unsigned short list[WIDE_WARPS][TAB / 2];
  u32 cnt[WIDE_WARPS];
};

template <int KIND, u32 TAB>
__global__ void __launch_bounds__(WIDE_WARPS * 32) k_eval_wide(EvalArgs A) {
  extern __shared__ __align__(16) unsigned char wide_raw[];
  WideSmem<TAB>& W = *reinterpret_cast<WideSmem<TAB>*>(wide_raw);
  const u32 lane = threadIdx.x & 31;
  const u32 wib = threadIdx.x >> 5;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  unsigned long long trav = 0, ncand = 0;
  u32* tk = W.tk[wib];
  unsigned short* tp = W.tp[wib];
  double* tv = W.tv[wib];
  unsigned short* list = W.list[wib];
  double* sw = W.sw[wib];
  for (u32 x = lane; x < TAB; x += 32) tk[x] = NONE32;
  __syncwarp();
  // The next vertex's list entry, id and row bounds are loaded one step at a
  // time while this vertex is folded, so that its row loads can start at once.
  u32 i_nx = 0, v_nx = 0;
  u64 o0_nx = 0, o1_nx = 0;
  if (warp < A.nidx) {
    i_nx = A.idx[warp];
    v_nx = A.verts[i_nx];
    o0_nx = A.off[v_nx];
    o1_nx = A.off[v_nx + 1];
  }
  for (u64 t = warp; t < A.nidx; t += nwarps) {
    const u32 i = i_nx;
    const u32 v = v_nx;
    const u64 o0 = o0_nx, o1 = o1_nx;
    const u64 deg = o1 - o0;
    const bool has_nx = t + nwarps < A.nidx;
    if (has_nx) i_nx = A.idx[t + nwarps];
    const u32 fv = A.f[v];
    const u32 cur = (KIND == EVAL_MOVE) ? fv : A.s[v];
    const double kv = A.kdeg[v];
    const double dcur = A.d[cur];
    if (lane == 0) {
      trav += deg;
      W.cnt[wib] = 0;
    }
    u32 cap = 64;
    while (cap < 2 * deg) cap <<= 1;
    const u32 mask = cap - 1;
    __syncwarp();
    for (u64 b0 = o0; b0 < o1; b0 += WIDE_BATCH * 32) {
      u32 key[WIDE_BATCH];
#pragma unroll
      for (u32 j = 0; j < WIDE_BATCH; ++j) {
        u64 q = b0 + j * 32 + lane;
        key[j] = NONE32;
        double wv = 0.0;
        if (q < o1) {
          u32 nb = A.col[q];
          wv = A.w[q];
          if (!entry_key<KIND>(A, v, nb, fv, key[j])) key[j] = NONE32;
        }
        sw[j * 32 + lane] = wv;
      }
      __syncwarp();
#pragma unroll
      for (u32 j = 0; j < WIDE_BATCH; ++j) {
        if (b0 + j * 32 >= o1) break;
        u32 grp = __match_any_sync(0xffffffffu, key[j]);
        if (key[j] != NONE32 && lane == (u32)(__ffs(grp) - 1)) {
          u32 slot = hash32(key[j]) & mask;
          u32 prev;
          while (true) {
            prev = atomicCAS(&tk[slot], NONE32, key[j]);
            if (prev == NONE32 || prev == key[j]) break;
            slot = (slot + 1) & mask;
          }
          double acc = prev == NONE32 ? 0.0 : tv[slot];
          for (u32 m = grp; m; m &= m - 1) acc = __dadd_rn(acc, sw[j * 32 + __ffs(m) - 1]);
          tv[slot] = acc;
          if (prev == NONE32) {
            tp[slot] = (unsigned short)(b0 + j * 32 + lane - o0);
            list[atomicAdd(&W.cnt[wib], 1u)] = (unsigned short)slot;
          }
        }
        __syncwarp();
      }
    }
    if (has_nx) v_nx = A.verts[i_nx];
    const u32 used = W.cnt[wib];
    // w(v, cur), then the argmax over the used slots, resetting them.
    double wcur = 0.0;
    bool found = false;
    for (u32 x = lane; x < used; x += 32) {
      u32 sl = list[x];
      if (tk[sl] == cur) {
        wcur = tv[sl];
        found = true;
      }
    }
    u32 fm = __ballot_sync(0xffffffffu, found);
    wcur = __shfl_sync(0xffffffffu, wcur, fm ? __ffs(fm) - 1 : 0);
    if (!fm) wcur = 0.0;
    __syncwarp();
    if (has_nx) {
      o0_nx = A.off[v_nx];
      o1_nx = A.off[v_nx + 1];
    }
    double g = -1.0;
    u32 p = NONE32, kk = cur;
    GainScreen scr;  // exact gains only for candidates that may win
    scr.init(wcur, A.tw, A.gamma, kv, dcur);
    for (u32 x0 = lane; x0 < used; x0 += 32 * WIDE_SCAN_UNROLL) {
      u32 key[WIDE_SCAN_UNROLL], sl[WIDE_SCAN_UNROLL];
      double dk[WIDE_SCAN_UNROLL];
#pragma unroll
      for (u32 j = 0; j < WIDE_SCAN_UNROLL; ++j) {
        const u32 x = x0 + 32 * j;
        sl[j] = x < used ? list[x] : 0u;
        key[j] = x < used ? tk[sl[j]] : NONE32;
        if (x < used) tk[sl[j]] = NONE32;
        if (key[j] == cur || A.tw == 0.0) key[j] = NONE32;
        if (KIND == EVAL_REFINE && key[j] != NONE32 && A.blocked[key[j]]) key[j] = NONE32;
      }
#pragma unroll
      for (u32 j = 0; j < WIDE_SCAN_UNROLL; ++j) dk[j] = key[j] != NONE32 ? A.d[key[j]] : 0.0;
#pragma unroll
      for (u32 j = 0; j < WIDE_SCAN_UNROLL; ++j) {
        if (key[j] == NONE32) continue;
        ++ncand;
        if (!scr.keep(tv[sl[j]], dk[j])) continue;
        const double gn = move_gain(tv[sl[j]], wcur, A.tw, A.gamma, kv, dcur, dk[j]);
        const u32 pp = tp[sl[j]];
        if (p == NONE32 || gn > g || (gn == g && pp < p)) {
          g = gn;
          p = pp;
          kk = key[j];
        }
      }
    }
    for (int o = 16; o; o >>= 1) {
      double og = __shfl_xor_sync(0xffffffffu, g, o);
      u32 op = __shfl_xor_sync(0xffffffffu, p, o);
      u32 ok = __shfl_xor_sync(0xffffffffu, kk, o);
      if (op != NONE32 && (p == NONE32 || og > g || (og == g && op < p))) {
        g = og;
        p = op;
        kk = ok;
      }
    }
    if (lane == 0) finish<KIND>(A, i, v, cur, kv, wcur, g, kk, p != NONE32);
    __syncwarp();
  }
  block_count(A, trav, ncand);
}

// ---------------------------------------------------------------------------
// Large degrees (> WIDE_MAX): a block per vertex.
//
// The row streams through in tiles of BIG_THREADS entries with a two-stage
// software pipeline: while tile t is folded, the keys of tile t+1 are being
// gathered and the neighbours and weights of tile t+2 loaded.  Each tile is
// bucketed (stable) by a hash partition of its keys, one partition per warp,
// so a warp folds exactly the entries of its own keys, in CSR order, and no
// key is touched by two warps: every key's sum is extended in the reference's
// order and rounding with no atomics on values.  Inside a warp the lanes that
// share a key are grouped with match_any; all group leaders fold their groups
// at once in one unrolled pass over the chunk.  With integral weights (sums
// exact in any order) there is no bucketing: each warp inserts its lanes'
// entries with atomics, one barrier per tile.
//
// The bin is ordered by degree and vertices are handed out largest first
// through a work counter.  The table lives in shared memory (BIG_TAB slots):
// hubs have long rows but few distinct neighbour keys.  A launch without
// global regions (pass 1) defers a row that passes BIG_TAB / 2 distinct keys
// to an overflow list; pass 2 takes those rows on blocks that own global
// regions, moving a row's table there when it passes the same bound.
// ---------------------------------------------------------------------------
constexpr u32 BIG_TAB = 4096;
constexpr u32 BIG_SCAN_UNROLL = 4;  // table slots a thread scans at a time
// Used-slot list of the shared table: a row is checked against BIG_TAB / 2
// distinct keys after every tile, so it holds at most that plus one tile's
constexpr u32 BIG_LIST = BIG_TAB / 2 + BIG_THREADS;
constexpr u64 BIG_DIRECT_DEFER = 2 * BIG_TAB;  // integral weights: longer rows are deferred unread
// (the autotuner may pick another bound; see HUB_DEFER_CAND)
constexpr u32 BIG_WARPS = BIG_THREADS / 32;
constexpr u32 BIG_PART_BITS = 3;  // log2(BIG_WARPS)
static_assert((1u << BIG_PART_BITS) == BIG_WARPS, "one key partition per warp");

template <int KIND>
__device__ __forceinline__ u32 tile_key(const EvalArgs& A, u32 v, u32 fv, bool ok, u32 nb) {
  u32 key = NONE32;
  if (ok && !entry_key<KIND>(A, v, nb, fv, key)) key = NONE32;
  return key;
}

// Find or claim the slot of `key` (linear probing; free slots hold NONE32).
__device__ __forceinline__ u64 claim_slot(u32* tk, u64 mask, u32 key, bool& fresh) {
  u64 slot = hash32(key) & mask;
  while (true) {
    u32 prev = atomicCAS(&tk[slot], NONE32, key);
    if (prev == NONE32) {
      fresh = true;
      return slot;
    }
    if (prev == key) {
      fresh = false;
      return slot;
    }
    slot = (slot + 1) & mask;
  }
}

// A table value of the block kernel: a double, or with integral weights the
// bits of an exact integer sum (added with 64-bit integer atomics).
__device__ __forceinline__ double tab_value(double raw, bool integer) {
  if (!integer) return raw;
  return dbl_of((unsigned long long)__double_as_longlong(raw));
}

template <int KIND>
__global__ void __launch_bounds__(BIG_THREADS) k_eval_big(EvalArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* s_tv = reinterpret_cast<double*>(smem_raw);        // BIG_TAB values
  u32* s_tk = reinterpret_cast<u32*>(s_tv + BIG_TAB);        // BIG_TAB keys
  u32* s_tp = s_tk + BIG_TAB;                                // BIG_TAB first positions
  double* b_w = reinterpret_cast<double*>(s_tp + BIG_TAB);   // bucketed tile: weights
  u32* b_key = reinterpret_cast<u32*>(b_w + BIG_THREADS);    // keys
  u32* b_pos = b_key + BIG_THREADS;                          // positions in the row
  // used slots of the shared table, in insertion order (the scan visits and
  // resets only these)
  unsigned short* s_list = reinterpret_cast<unsigned short*>(b_pos + BIG_THREADS);
  __shared__ u32 s_cnt[BIG_WARPS * BIG_WARPS];               // [partition][warp]
  __shared__ u32 s_off[BIG_WARPS * BIG_WARPS + 1];
  __shared__ double r_g[BIG_WARPS];
  __shared__ u32 r_p[BIG_WARPS], r_k[BIG_WARPS];
  __shared__ double s_wcur;
  __shared__ u32 s_used, s_gused, s_next;
  const u32 tid = threadIdx.x;
  const u32 lane = tid & 31;
  const u32 wib = tid >> 5;
  const u32 lt_mask = (1u << lane) - 1u;
  unsigned long long trav = 0, ncand = 0;
  u32* g_tk = A.tkey ? A.tkey + (u64)blockIdx.x * A.region : nullptr;
  u32* g_tp = A.tpos ? A.tpos + (u64)blockIdx.x * A.region : nullptr;
  double* g_tv = A.tval ? A.tval + (u64)blockIdx.x * A.region : nullptr;
  u32* g_list = A.tlist ? A.tlist + (u64)blockIdx.x * (A.region / 2) : nullptr;
  const u32 nidx = A.nidx_dev ? *A.nidx_dev : A.nidx;
  // the shared table starts clean; each row resets the slots it used
  for (u32 x = tid; x < BIG_TAB; x += BIG_THREADS) {
    s_tk[x] = NONE32;
    s_tv[x] = 0.0;
    s_tp[x] = NONE32;
  }
  // Vertices are taken from a shared counter (the list is ordered by degree,
  // largest first), so the longest rows start first and no block queues
  // several of them behind each other.
  for (;;) {
    if (tid == 0) s_next = atomicAdd(A.work, 1u);
    __syncthreads();
    const u32 t = s_next;
    if (t >= nidx) break;
    const u32 i = A.idx[t];
    const u32 v = A.verts[i];
    const u64 o0 = A.off[v], o1 = A.off[v + 1];
    const u64 deg = o1 - o0;
    const u32 fv = A.f[v];
    const u32 cur = (KIND == EVAL_MOVE) ? fv : A.s[v];
    const double kv = A.kdeg[v];
    // Integral weights: a row this long goes straight to the partitioned
    // pass (it almost always passes BIG_TAB / 2 distinct keys, found only
    // after part of the row has been folded).
    if (A.defer_deg && !g_tk && deg > A.defer_deg) {
      if (tid == 0) A.ovf_list[atomicAdd(A.ovf_count, 1u)] = i;
      __syncthreads();
      continue;
    }
    u64 gcap = 64;
    while (gcap < 2 * deg) gcap <<= 1;
    const u32 cap = gcap < BIG_TAB ? (u32)gcap : BIG_TAB;
    if (tid == 0) {
      s_used = 0;
      s_gused = 0;
    }
    // pipeline prologue: keys of tile 0, neighbours of tile 1
    u32 key1;
    double w1 = 0.0;
    {
      const u64 q = o0 + tid;
      const bool ok = q < o1;
      const u32 nb = ok ? A.col[q] : 0u;
      w1 = ok ? A.w[q] : 0.0;
      key1 = tile_key<KIND>(A, v, fv, ok, nb);
    }
    u32 nb2 = 0;
    double w2 = 0.0;
    bool ok2;
    {
      const u64 q = o0 + BIG_THREADS + tid;
      ok2 = q < o1;
      if (ok2) {
        nb2 = A.col[q];
        w2 = A.w[q];
      }
    }
    bool global = false;
    bool deferred = false;
    u32* tk = s_tk;
    u32* tp = s_tp;
    double* tv = s_tv;
    u64 mask = cap - 1;
    __syncthreads();
    for (u64 b0 = o0; b0 < o1; b0 += BIG_THREADS) {
      const u32 key = key1;
      const double wv = w1;
      const u32 pos = (u32)(b0 - o0) + tid;
      // advance the pipeline: gather tile t+1's keys, load tile t+2's entries
      key1 = tile_key<KIND>(A, v, fv, ok2, nb2);
      w1 = w2;
      {
        const u64 q = b0 + 2 * BIG_THREADS + tid;
        ok2 = q < o1;
        nb2 = ok2 ? A.col[q] : 0u;
        w2 = ok2 ? A.w[q] : 0.0;
      }
      // stable bucketing of the tile by key partition (ordered sums only)
      const u32 part = key == NONE32 ? NONE32 : hash32(key) >> (32 - BIG_PART_BITS);
      u32 rank = 0, mycnt = 0;
      if (!A.concurrent) {
#pragma unroll
        for (u32 q = 0; q < BIG_WARPS; ++q) {
          const u32 bq = __ballot_sync(0xffffffffu, part == q);
          if (lane == q) mycnt = __popc(bq);
          if (part == q) rank = __popc(bq & lt_mask);
        }
        if (lane < BIG_WARPS) s_cnt[lane * BIG_WARPS + wib] = mycnt;
      }
      __syncthreads();
      // The previous tile's folds are complete here and s_used is stable.  A
      // row with too many distinct keys moves its table to the block's global
      // region; a launch without regions defers the row to its overflow list
      // instead (a later launch with regions takes it from the start).
      if (!global && s_used > BIG_TAB / 2 && !g_tk) {
        deferred = true;
        break;
      }
      if (!global && s_used > BIG_TAB / 2) {
        // the used shared slots move to the global table and are reset
        const u64 gmask = gcap - 1;
        const u32 nu = s_used;
        for (u32 x = tid; x < nu; x += BIG_THREADS) {
          const u32 sx = s_list[x];
          bool fresh;
          const u64 sl = claim_slot(g_tk, gmask, s_tk[sx], fresh);
          g_tv[sl] = s_tv[sx];
          g_tp[sl] = s_tp[sx];
          g_list[atomicAdd(&s_gused, 1u)] = (u32)sl;
          s_tk[sx] = NONE32;
          s_tv[sx] = 0.0;
          s_tp[sx] = NONE32;
        }
        global = true;
        tk = g_tk;
        tp = g_tp;
        tv = g_tv;
        mask = gmask;
        // every moved slot is written before any entry is added to it
        __syncthreads();
      }
      if (A.concurrent) {
        // Integral weights: every order of additions gives the same sums, so
        // each warp inserts its own lanes' entries right away, lanes sharing a
        // key combined first; the first position is the smallest one.
        const bool okk = key != NONE32;
        const u32 grp = __match_any_sync(0xffffffffu, okk ? (unsigned long long)key
                                                           : ((1ull << 32) | lane));
        const bool leader = okk && lane == (u32)(__ffs(grp) - 1);
        // the group's integer sum: a lane alone in its group has it already;
        // otherwise its leader adds the group up from shared memory
        unsigned long long isum = okk ? int_of(wv) : 0ull;
        if (__all_sync(0xffffffffu, isum < (1ull << 26))) {
          u32 pdummy;
          group_sums(grp, lane, okk, (u32)isum, 0u, isum, pdummy);
        } else if (!__all_sync(0xffffffffu, (grp & (grp - 1)) == 0)) {
          b_w[tid] = wv;
          __syncwarp();
          if (leader) {
            double gsum = 0.0;
            for (u32 m = grp; m; m &= m - 1) gsum += b_w[(tid & ~31u) + __ffs(m) - 1];
            isum = int_of(gsum);
          }
          __syncwarp();
        }
        bool fresh = false;
        u64 slot = 0;
        if (leader) {
          slot = claim_slot(tk, mask, key, fresh);
          if (fresh && global) g_list[atomicAdd(&s_gused, 1u)] = (u32)slot;
          // the slot holds the integer sum (0.0 and integer 0 share their bits);
          // the leader's position is the group's first
          atomicAdd(reinterpret_cast<unsigned long long*>(&tv[slot]), isum);
          atomicMin(&tp[slot], pos);
        }
        if (!global) {
          const u32 fm = __ballot_sync(0xffffffffu, fresh);
          if (fm) {
            u32 at = 0;
            if (lane == 0) at = atomicAdd(&s_used, (u32)__popc(fm));
            at = __shfl_sync(0xffffffffu, at, 0);
            if (fresh) s_list[at + __popc(fm & lt_mask)] = (unsigned short)slot;
          }
        }
        __syncwarp();
        continue;
      }
      if (wib == 0) {
        // exclusive scan of the 64 counts in (partition, warp) order
        const u32 a0 = s_cnt[2 * lane], a1 = s_cnt[2 * lane + 1];
        u32 inc = a0 + a1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const u32 y = __shfl_up_sync(0xffffffffu, inc, o);
          if (lane >= (u32)o) inc += y;
        }
        const u32 ex = inc - a0 - a1;
        s_off[2 * lane] = ex;
        s_off[2 * lane + 1] = ex + a0;
        if (lane == 31) s_off[BIG_WARPS * BIG_WARPS] = inc;
      }
      __syncthreads();
      if (part != NONE32) {
        const u32 dst = s_off[part * BIG_WARPS + wib] + rank;
        b_key[dst] = key;
        b_w[dst] = wv;
        b_pos[dst] = pos;
      }
      const u32 beg = s_off[wib * BIG_WARPS];
      const u32 end = s_off[(wib + 1) * BIG_WARPS];
      __syncthreads();
      // this warp's keys, in CSR order
      for (u32 c = beg; c < end; c += 32) {
        const u32 e = c + lane;
        const bool ok = e < end;
        const u32 k = ok ? b_key[e] : NONE32;
        const u32 grp = __match_any_sync(0xffffffffu, ok ? (unsigned long long)k
                                                         : ((1ull << 32) | lane));
        const bool leader = ok && lane == (u32)(__ffs(grp) - 1);
        u64 slot = 0;
        double acc = 0.0;
        if (leader) {
          bool fresh;
          slot = claim_slot(tk, mask, k, fresh);
          if (fresh) {
            tp[slot] = b_pos[e];
            if (global) g_list[atomicAdd(&s_gused, 1u)] = (u32)slot;
            else s_list[atomicAdd(&s_used, 1u)] = (unsigned short)slot;
          }
          acc = tv[slot];
        }
        const u32 nhere = end - c < 32 ? end - c : 32;
#pragma unroll
        for (u32 j = 0; j < 32; ++j) {
          if (j < nhere) {
            const double y = b_w[c + j];
            if (leader && ((grp >> j) & 1u)) acc = __dadd_rn(acc, y);
          }
        }
        if (leader) tv[slot] = acc;
        __syncwarp();
      }
    }
    if (deferred) {
      const u32 nu = s_used;  // stable: the loop left right after a barrier
      for (u32 x = tid; x < nu; x += BIG_THREADS) {
        const u32 sx = s_list[x];
        s_tk[sx] = NONE32;
        s_tv[sx] = 0.0;
        s_tp[sx] = NONE32;
      }
      if (tid == 0) A.ovf_list[atomicAdd(A.ovf_count, 1u)] = i;
      __syncthreads();
      continue;
    }
    __syncthreads();
    // w(v, cur), then the argmax over the used slots (each reset after it is read).
    if (tid == 0) {
      double wc = 0.0;
      u64 sl = hash32(cur) & mask;
      while (tk[sl] != NONE32) {
        if (tk[sl] == cur) {
          wc = tab_value(tv[sl], A.concurrent);
          break;
        }
        sl = (sl + 1) & mask;
      }
      s_wcur = wc;
    }
    __syncthreads();
    const double wcur = s_wcur;
    const double dcur = A.d[cur];
    const u32 nscan = global ? s_gused : s_used;
    double g = -1.0;
    u32 p = NONE32, kk = cur;
    // BIG_SCAN_UNROLL slots per thread at a time: their community degrees
    // are gathered together
    GainScreen scr;  // exact gains only for candidates that may win
    scr.init(wcur, A.tw, A.gamma, kv, dcur);
    for (u32 x0 = tid; x0 < nscan; x0 += BIG_THREADS * BIG_SCAN_UNROLL) {
      u32 key[BIG_SCAN_UNROLL], pq[BIG_SCAN_UNROLL];
      double val[BIG_SCAN_UNROLL], dk[BIG_SCAN_UNROLL];
#pragma unroll
      for (u32 j = 0; j < BIG_SCAN_UNROLL; ++j) {
        const u32 x = x0 + j * BIG_THREADS;
        key[j] = NONE32;
        if (x >= nscan) continue;
        const u64 sl = global ? g_list[x] : s_list[x];
        key[j] = tk[sl];
        if (key[j] == NONE32) continue;
        val[j] = tab_value(tv[sl], A.concurrent);
        pq[j] = tp[sl];
        tk[sl] = NONE32;
        tv[sl] = 0.0;
        tp[sl] = NONE32;
        if (key[j] == cur || A.tw == 0.0) key[j] = NONE32;
        else if (KIND == EVAL_REFINE && A.blocked[key[j]]) key[j] = NONE32;
      }
#pragma unroll
      for (u32 j = 0; j < BIG_SCAN_UNROLL; ++j) dk[j] = key[j] != NONE32 ? A.d[key[j]] : 0.0;
#pragma unroll
      for (u32 j = 0; j < BIG_SCAN_UNROLL; ++j) {
        if (key[j] == NONE32) continue;
        ++ncand;
        if (!scr.keep(val[j], dk[j])) continue;
        const double gn = move_gain(val[j], wcur, A.tw, A.gamma, kv, dcur, dk[j]);
        if (p == NONE32 || gn > g || (gn == g && pq[j] < p)) {
          g = gn;
          p = pq[j];
          kk = key[j];
        }
      }
    }
    for (int o = 16; o; o >>= 1) {
      const double og = __shfl_xor_sync(0xffffffffu, g, o);
      const u32 op = __shfl_xor_sync(0xffffffffu, p, o);
      const u32 ok = __shfl_xor_sync(0xffffffffu, kk, o);
      if (op != NONE32 && (p == NONE32 || og > g || (og == g && op < p))) {
        g = og;
        p = op;
        kk = ok;
      }
    }
    if (lane == 0) {
      r_g[wib] = g;
      r_p[wib] = p;
      r_k[wib] = kk;
    }
    __syncthreads();
    if (tid == 0) {
      for (u32 x = 1; x < BIG_WARPS; ++x) {
        if (r_p[x] != NONE32 && (p == NONE32 || r_g[x] > g || (r_g[x] == g && r_p[x] < p))) {
          g = r_g[x];
          p = r_p[x];
          kk = r_k[x];
        }
      }
      trav += deg;
      finish<KIND>(A, i, v, cur, kv, wcur, g, kk, p != NONE32);
    }
    __syncthreads();
  }
  block_count(A, trav, ncand);
}

// ---------------------------------------------------------------------------
// Second pass for integral weights: the rows deferred by pass 1 (long rows,
// or more than BIG_TAB / 2 distinct keys) are hash-partitioned into buckets
// that fit a warp's shared-memory table, so that every warp of the GPU folds
// one bucket instead of a few blocks walking global tables.  Integral sums are exact in
// any order, and a key's first CSR position is the minimum of its entries'
// positions, so neither the partition order nor the fold order matters.
//   plan     per row: buckets B = 2^k >= deg / PB_TARGET, 4096-entry chunks;
//   hist     per chunk: each entry's key (saved), its bucket's count, and the
//            row's w(v, cur);
//   scatter  per chunk: (key, position, weight) into its bucket's range;
//   fold     per bucket: a warp's shared table, then the bucket's best candidate;
//   final    per row: the best over its buckets, then the empty community.
// A bucket holds at most about PB_TARGET entries plus the repeats of its
// keys (a heavy key adds entries, not keys), so its distinct keys fit a
// table of 2 x PB_TARGET slots.  A bucket whose keys fill its table (far out
// in the tail of the hash spread) fails its row, which then takes the
// global-table pass.
// ---------------------------------------------------------------------------
constexpr u32 PB_TARGET = 256;  // expected entries per bucket
constexpr u32 PB_TAB = 512;     // table slots of a fold warp
constexpr u32 PB_CHUNK = 4096;   // entries per block of the hist / scatter kernels
constexpr u32 PB_HIST = 8192;    // buckets a block counts in shared memory
constexpr u32 PB_FOLD_UNROLL = 4;  // chunks (or table slots) a fold thread has in flight

__global__ void k_pb_plan(const u32* ovf, const u32* novf, const u32* verts, const u64* off,
                          u32* nb, u64* ne, u32* nc) {
  const u32 m = *novf;
  for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < m; t += (u64)gridDim.x * blockDim.x) {
    const u32 v = verts[ovf[t]];
    const u64 d = off[v + 1] - off[v];
    u32 b = 1;
    while ((u64)b * PB_TARGET < d) b <<= 1;
    nb[t] = b;
    ne[t] = d;
    nc[t] = (u32)((d + PB_CHUNK - 1) / PB_CHUNK);
  }
}

// Bucket of a key among B = 2^k buckets: the top k bits of its hash.  The
// fold kernel's table slot takes the low bits of the same hash, so a bucket's
// keys still spread over the whole table.
__device__ __forceinline__ u32 pb_bucket(u32 key, u32 B) {
  return B <= 1 ? 0u : hash32(key) >> (32 - (__ffs(B) - 1));
}

struct PbArgs {
  const u32* border;   // the round's buckets, most entries first (fold order)
  u32* fold_work;      // next position of border a fold block takes
  const u32* ovf;      // deferred idx values
  const u32* nb;       // buckets per row
  const u64* ebase;    // exclusive scan of row degrees
  const u32* bbase;    // exclusive scan of bucket counts
  const u32* cbase;    // exclusive scan of chunk counts
  u32 r0, r1;          // rows of this round
  u64 e0;              // ebase[r0]
  u32 b0, c0, c1;      // bbase[r0], cbase[r0], the round's end chunk
  u32* ktmp;           // entry keys (NONE32: skipped)
  u32* bcnt;           // per bucket: count, then scatter cursor
  u32* boff;           // per bucket: first entry (exclusive scan of bcnt)
  u32* ekey;
  u32* epos;
  double* ew;
  double* wcur;        // per row w(v, cur)
  double* bg;          // per bucket best gain, position, key
  u32* bp;
  u32* bk;
  u32* rowfail;        // per row: a bucket overflowed
  // filled once per pass by k_pb_rows, so that no kernel searches for its row
  // or walks idx -> vertex -> label -> degree before its real work
  const u32* brow;     // global bucket -> row
  const u32* crow;     // global chunk -> row
  const u32* rv;       // per row: vertex, f[v], its current label, k_v, d[cur], off[v]
  const u32* rfv;
  const u32* rcur;
  const double* rkv;
  const double* rdcur;
  const u64* ro0;
  const u64* ne;       // per row: degree
};

// Sort keys of the fold order: each bucket's entry count, and its index.
__global__ void k_pb_order_keys(const u32* boff, u32 nb, u32* key, u32* val) {
  for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < nb; t += (u64)gridDim.x * blockDim.x) {
    key[t] = boff[t + 1] - boff[t];
    val[t] = (u32)t;
  }
}

// Per row of the pass: its scalars, and its entries in the bucket -> row and
// chunk -> row maps (a warp per row).
template <int KIND>
__global__ void k_pb_rows(EvalArgs A, const u32* ovf, u32 m, const u32* nb, const u32* bbase,
                          const u32* nc, const u32* cbase, u32* brow, u32* crow, u32* rv, u32* rfv,
                          u32* rcur, double* rkv, double* rdcur, u64* ro0) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 r = warp; r < m; r += nwarps) {
    if (lane == 0) {
      const u32 v = A.verts[ovf[r]];
      const u32 fv = A.f[v];
      const u32 cur = (KIND == EVAL_MOVE) ? fv : A.s[v];
      rv[r] = v;
      rfv[r] = fv;
      rcur[r] = cur;
      rkv[r] = A.kdeg[v];
      rdcur[r] = A.d[cur];
      ro0[r] = A.off[v];
    }
    const u32 b0 = bbase[r], b1 = b0 + nb[r];
    for (u32 x = b0 + lane; x < b1; x += 32) brow[x] = (u32)r;
    const u32 c0 = cbase[r], c1 = c0 + nc[r];
    for (u32 x = c0 + lane; x < c1; x += 32) crow[x] = (u32)r;
  }
}

template <int KIND>
__global__ void __launch_bounds__(256) k_pb_hist(EvalArgs A, PbArgs P) {
  __shared__ u32 s_hist[PB_HIST];
  __shared__ double s_red[8];
  for (u32 c = P.c0 + blockIdx.x; c < P.c1; c += gridDim.x) {
    const u32 r = P.crow[c];
    const u32 v = P.rv[r];
    const u64 o0 = P.ro0[r], o1 = o0 + P.ne[r];
    const u64 lo = o0 + (u64)(c - P.cbase[r]) * PB_CHUNK;
    const u64 hi = lo + PB_CHUNK < o1 ? lo + PB_CHUNK : o1;
    const u32 fv = P.rfv[r];
    const u32 cur = P.rcur[r];
    const u32 B = P.nb[r];
    const bool local = B <= PB_HIST;
    u32* gcnt = P.bcnt + (P.bbase[r] - P.b0);
    if (local)
      for (u32 x = threadIdx.x; x < B; x += blockDim.x) s_hist[x] = 0;
    __syncthreads();
    double wc = 0.0;
    const u64 ebase = P.ebase[r] - P.e0 + (lo - o0);
    const u32 lane = threadIdx.x & 31;
    // PB_FOLD_UNROLL entries per thread in flight (neighbours, then their
    // keys); lanes counting into the same bucket add once
    for (u64 w0 = lo + (threadIdx.x & ~31u); w0 < hi; w0 += 256 * PB_FOLD_UNROLL) {
      u32 nb[PB_FOLD_UNROLL], key[PB_FOLD_UNROLL];
#pragma unroll
      for (u32 j = 0; j < PB_FOLD_UNROLL; ++j) {
        const u64 q = w0 + j * 256 + lane;
        nb[j] = q < hi ? A.col[q] : NONE32;
      }
#pragma unroll
      for (u32 j = 0; j < PB_FOLD_UNROLL; ++j) {
        key[j] = NONE32;
        if (nb[j] != NONE32 && !entry_key<KIND>(A, v, nb[j], fv, key[j])) key[j] = NONE32;
      }
#pragma unroll
      for (u32 j = 0; j < PB_FOLD_UNROLL; ++j) {
        const u64 q = w0 + j * 256 + lane;
        if (q < hi) P.ktmp[ebase + (q - lo)] = key[j];
        const bool ok = key[j] != NONE32;
        if (ok && key[j] == cur) wc += A.w[q];
        const u32 b = ok ? pb_bucket(key[j], B) : 0u;
        const u32 grp = __match_any_sync(0xffffffffu, ok ? (unsigned long long)b
                                                         : ((1ull << 32) | lane));
        if (ok && lane == (u32)(__ffs(grp) - 1)) {
          if (local) atomicAdd(&s_hist[b], (u32)__popc(grp));
          else atomicAdd(&gcnt[b], (u32)__popc(grp));
        }
      }
    }
    for (int o = 16; o; o >>= 1) wc += __shfl_xor_sync(0xffffffffu, wc, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = wc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (u32 x = 0; x < blockDim.x / 32; ++x) t += s_red[x];
      if (t != 0.0) atomicAdd(&P.wcur[r], t);  // integral: exact in any order
    }
    if (local)
      for (u32 x = threadIdx.x; x < B; x += blockDim.x)
        if (s_hist[x]) atomicAdd(&gcnt[x], s_hist[x]);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) k_pb_scatter(EvalArgs A, PbArgs P) {
  const u32 lane = threadIdx.x & 31;
  for (u32 c = P.c0 + blockIdx.x; c < P.c1; c += gridDim.x) {
    const u32 r = P.crow[c];
    const u64 o0 = P.ro0[r], o1 = o0 + P.ne[r];
    const u64 lo = o0 + (u64)(c - P.cbase[r]) * PB_CHUNK;
    const u64 hi = lo + PB_CHUNK < o1 ? lo + PB_CHUNK : o1;
    const u32 B = P.nb[r];
    u32* cursor = P.bcnt + (P.bbase[r] - P.b0);
    const u32* start = P.boff + (P.bbase[r] - P.b0);
    const u64 ebase = P.ebase[r] - P.e0 + (lo - o0);
    // PB_FOLD_UNROLL entries per thread in flight; lanes bound for the same
    // bucket take their slots with one atomic (a heavy key fills one bucket)
    for (u64 w0 = lo + (threadIdx.x & ~31u); w0 < hi; w0 += 256 * PB_FOLD_UNROLL) {
      const u64 q0 = w0 + lane;
      u32 key[PB_FOLD_UNROLL];
      double wq[PB_FOLD_UNROLL];
#pragma unroll
      for (u32 j = 0; j < PB_FOLD_UNROLL; ++j) {
        const u64 q = q0 + j * 256;
        key[j] = q < hi ? P.ktmp[ebase + (q - lo)] : NONE32;
        wq[j] = key[j] != NONE32 ? A.w[q] : 0.0;
      }
#pragma unroll
      for (u32 j = 0; j < PB_FOLD_UNROLL; ++j) {
        const u64 q = q0 + j * 256;
        const bool ok = key[j] != NONE32;
        const u32 b = ok ? pb_bucket(key[j], B) : 0u;
        const u32 grp = __match_any_sync(0xffffffffu, ok ? (unsigned long long)b
                                                         : ((1ull << 32) | lane));
        const u32 leader = __ffs(grp) - 1;
        u32 at = 0;
        if (ok && lane == leader) at = start[b] + atomicAdd(&cursor[b], (u32)__popc(grp));
        at = __shfl_sync(0xffffffffu, at, leader);
        if (ok) {
          const u32 slot = at + __popc(grp & ((1u << lane) - 1u));
          P.ekey[slot] = key[j];
          P.epos[slot] = (u32)(q - o0);
          P.ew[slot] = wq[j];
        }
      }
    }
    __syncthreads();
  }
}

constexpr u32 PB_FOLD_WARPS = 4;  // warps of a fold block, one bucket each
constexpr size_t PB_FOLD_SMEM = (size_t)PB_FOLD_WARPS * PB_TAB * (8 + 4 + 4 + 2);

// Table slots the fold kernel may use (hl_dbg_set_bucket_slots lowers it so
// that tests reach the overflow path).
std::atomic<u32> g_pb_slots{PB_TAB};

// Hub-row deferral bound forced by hl_dbg_set_hub_defer (0: the handle's).
std::atomic<u32> g_dbg_hub_defer{0};

// One bucket per warp at a time, taken largest first from a shared counter
// (a hub's heavy-key bucket, a large community holding much of its row,
// starts at once instead of trailing the launch).  Each warp owns a table
// in shared memory that starts clean; every key it inserts is appended to
// the warp's used-slot list, so the argmax scan and the reset visit only used
// slots, and no block barrier is needed anywhere.
template <int KIND>
__global__ void __launch_bounds__(PB_FOLD_WARPS * 32) k_pb_fold(EvalArgs A, PbArgs P,
                                                                u32 nbuckets, u32 tab_limit) {
  extern __shared__ __align__(16) unsigned char pb_smem[];
  __shared__ unsigned long long s_wb[PB_FOLD_WARPS][32];  // a chunk's weights, per warp
  __shared__ u32 s_pb[PB_FOLD_WARPS][32];                 // and positions
  const u32 lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  unsigned long long* tv = reinterpret_cast<unsigned long long*>(pb_smem) + (size_t)wib * PB_TAB;
  u32* tk = reinterpret_cast<u32*>(reinterpret_cast<unsigned long long*>(pb_smem) +
                                   (size_t)PB_FOLD_WARPS * PB_TAB) + (size_t)wib * PB_TAB;
  u32* tp = tk + (size_t)PB_FOLD_WARPS * PB_TAB;
  unsigned short* list = reinterpret_cast<unsigned short*>(
                             reinterpret_cast<u32*>(pb_smem + (size_t)PB_FOLD_WARPS * PB_TAB * 8) +
                             (size_t)2 * PB_FOLD_WARPS * PB_TAB) + (size_t)wib * PB_TAB;
  const u32 lt = (1u << lane) - 1u;
  unsigned long long ncand = 0;
  for (u32 x = lane; x < PB_TAB; x += 32) {
    tk[x] = NONE32;
    tp[x] = NONE32;
    tv[x] = 0ull;
  }
  __syncwarp();
  for (;;) {
    u32 item = 0;
    if (lane == 0) item = atomicAdd(P.fold_work, 1u);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= nbuckets) break;
    const u32 bl = P.border[item];
    const u32 r = P.brow[P.b0 + bl];
    const u32 e_lo = P.boff[bl], e_hi = P.boff[bl + 1];
    const u32 cnt = e_hi - e_lo;
    u32 cap = 64;
    while (cap < 2 * cnt && cap < tab_limit) cap <<= 1;
    const u32 mask = cap - 1;
    u32 nused = 0;
    bool ovf = false;
    // PB_FOLD_UNROLL chunks of 32 entries at a time, their loads issued
    // together.  Lanes of a chunk that share a key are combined first
    // (match_any), so a heavy key costs one table update per chunk.
    for (u32 base = e_lo; base < e_hi; base += 32 * PB_FOLD_UNROLL) {
      u32 ek[PB_FOLD_UNROLL], ep[PB_FOLD_UNROLL];
      unsigned long long ew[PB_FOLD_UNROLL];
#pragma unroll
      for (u32 j = 0; j < PB_FOLD_UNROLL; ++j) {
        const u32 e = base + j * 32 + lane;
        const bool ok = e < e_hi;
        ek[j] = ok ? P.ekey[e] : NONE32;
        ep[j] = ok ? P.epos[e] : NONE32;
        // integral weights: every partial sum is an exact integer
        ew[j] = ok ? int_of(P.ew[e]) : 0ull;
      }
#pragma unroll
      for (u32 j = 0; j < PB_FOLD_UNROLL; ++j) {
        if (base + j * 32 >= e_hi) break;  // warp-uniform
        const bool ok = ek[j] != NONE32;
        const u32 grp = __match_any_sync(0xffffffffu, ok ? (unsigned long long)ek[j]
                                                         : ((1ull << 32) | lane));
        const bool leader = ok && lane == (u32)(__ffs(grp) - 1);
        // the group's sum and first position: a lane alone in its group has
        // them already; otherwise its leader adds the group up from shared
        // memory (as many steps as the largest group of the chunk)
        unsigned long long sum = ew[j];
        u32 pmin = ep[j];
        if (__all_sync(0xffffffffu, ew[j] < (1ull << 26))) {
          group_sums(grp, lane, ok, (u32)ew[j], ep[j], sum, pmin);
        } else if (!__all_sync(0xffffffffu, (grp & (grp - 1)) == 0)) {
          s_wb[wib][lane] = ew[j];
          s_pb[wib][lane] = ep[j];
          __syncwarp();
          if (leader) {
            sum = 0;
            pmin = NONE32;
            for (u32 m = grp; m; m &= m - 1) {
              const u32 l = __ffs(m) - 1;
              sum += s_wb[wib][l];
              pmin = min(pmin, s_pb[wib][l]);
            }
          }
          __syncwarp();
        }
        bool fresh = false, failed = false;
        u32 slot = 0;
        if (leader) {
          slot = hash32(ek[j]) & mask;
          u32 probes = 0;
          bool ins = false;
          while (probes++ < cap) {
            const u32 prev = atomicCAS(&tk[slot], NONE32, ek[j]);
            if (prev == NONE32 || prev == ek[j]) {
              ins = true;
              fresh = prev == NONE32;
              break;
            }
            slot = (slot + 1) & mask;
          }
          if (ins) {
            tv[slot] += sum;  // one leader per key in the warp: no atomics needed
            tp[slot] = min(tp[slot], pmin);
          } else {
            failed = true;
          }
        }
        const u32 fm = __ballot_sync(0xffffffffu, fresh);
        if (fresh) list[nused + __popc(fm & lt)] = (unsigned short)slot;
        nused += __popc(fm);
        ovf |= __any_sync(0xffffffffu, failed);
        __syncwarp();
      }
    }
    double g = -1.0;
    u32 p = NONE32, kk = NONE32;
    const bool scan = !ovf && A.tw != 0.0;
    const u32 cur = P.rcur[r];
    const double kv = P.rkv[r];
    const double wcur = P.wcur[r];
    const double dcur = P.rdcur[r];
    GainScreen scr;  // exact gains only for candidates that may win
    scr.init(wcur, A.tw, A.gamma, kv, dcur);
    // the used slots, PB_FOLD_UNROLL per lane at a time (their community
    // degrees gathered together), each reset after it is read
    for (u32 x0 = lane; x0 < nused; x0 += 32 * PB_FOLD_UNROLL) {
      u32 key[PB_FOLD_UNROLL], pq[PB_FOLD_UNROLL];
      unsigned long long vq[PB_FOLD_UNROLL];
      double dk[PB_FOLD_UNROLL];
#pragma unroll
      for (u32 j = 0; j < PB_FOLD_UNROLL; ++j) {
        const u32 x = x0 + j * 32;
        key[j] = NONE32;
        if (x >= nused) continue;
        const u32 sl = list[x];
        key[j] = tk[sl];
        vq[j] = tv[sl];
        pq[j] = tp[sl];
        tk[sl] = NONE32;
        tv[sl] = 0ull;
        tp[sl] = NONE32;
        if (!scan || key[j] == cur) key[j] = NONE32;
        else if (KIND == EVAL_REFINE && A.blocked[key[j]]) key[j] = NONE32;
      }
#pragma unroll
      for (u32 j = 0; j < PB_FOLD_UNROLL; ++j) dk[j] = key[j] != NONE32 ? A.d[key[j]] : 0.0;
#pragma unroll
      for (u32 j = 0; j < PB_FOLD_UNROLL; ++j) {
        if (key[j] == NONE32) continue;
        const double val = dbl_of(vq[j]);
        ++ncand;
        if (!scr.keep(val, dk[j])) continue;
        const double gn = move_gain(val, wcur, A.tw, A.gamma, kv, dcur, dk[j]);
        if (p == NONE32 || gn > g || (gn == g && pq[j] < p)) {
          g = gn;
          p = pq[j];
          kk = key[j];
        }
      }
    }
    for (int o = 16; o; o >>= 1) {
      const double og = __shfl_xor_sync(0xffffffffu, g, o);
      const u32 op = __shfl_xor_sync(0xffffffffu, p, o);
      const u32 ok = __shfl_xor_sync(0xffffffffu, kk, o);
      if (op != NONE32 && (p == NONE32 || og > g || (og == g && op < p))) {
        g = og;
        p = op;
        kk = ok;
      }
    }
    if (lane == 0) {
      P.bg[bl] = g;
      P.bp[bl] = p;
      P.bk[bl] = kk;
      if (ovf) P.rowfail[r] = 1;
    }
    __syncwarp();
  }
  block_count(A, 0, ncand);
}

// One warp per row: the best over the row's buckets, then the decision.
template <int KIND>
__global__ void k_pb_final(EvalArgs A, PbArgs P, u32* fail_list, u32* fail_count) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  unsigned long long trav = 0;
  for (u64 r = P.r0 + warp; r < P.r1; r += nwarps) {
    const u32 i = P.ovf[r];
    if (P.rowfail[r]) {
      if (lane == 0) fail_list[atomicAdd(fail_count, 1u)] = i;
      continue;
    }
    const u32 v = A.verts[i];
    const u32 B = P.nb[r];
    const u32 bb = P.bbase[r] - P.b0;
    double g = -1.0;
    u32 p = NONE32, kk = NONE32;
    for (u32 x = lane; x < B; x += 32) {
      const u32 pp = P.bp[bb + x];
      if (pp == NONE32) continue;
      const double gn = P.bg[bb + x];
      if (p == NONE32 || gn > g || (gn == g && pp < p)) {
        g = gn;
        p = pp;
        kk = P.bk[bb + x];
      }
    }
    for (int o = 16; o; o >>= 1) {
      const double og = __shfl_xor_sync(0xffffffffu, g, o);
      const u32 op = __shfl_xor_sync(0xffffffffu, p, o);
      const u32 ok = __shfl_xor_sync(0xffffffffu, kk, o);
      if (op != NONE32 && (p == NONE32 || og > g || (og == g && op < p))) {
        g = og;
        p = op;
        kk = ok;
      }
    }
    if (lane == 0) {
      const u32 fv = A.f[v];
      const u32 cur = (KIND == EVAL_MOVE) ? fv : A.s[v];
      trav += A.off[v + 1] - A.off[v];
      finish<KIND>(A, i, v, cur, A.kdeg[v], P.wcur[r], g, kk, p != NONE32);
    }
  }
  block_count(A, trav, 0);
}

// ---------------------------------------------------------------------------
// Host side: bin the list by degree and launch the three kernels.
// ---------------------------------------------------------------------------
// Bins: 0-2 sub-warp (deg <= 8, 16, 32), 3 warp table (<= mid_max), 4 wide
// (<= WIDE_SPLIT), 6 wide (<= wide_max) with full-size tables, 5 block.
constexpr int NBINS = 7;

__global__ void k_bin(const u32* verts, u32 nv, const u64* off, u32* bin, u32* idx,
                      u32* counts, unsigned long long* maxdeg, u32 mid_max, u32 wide_max) {
  __shared__ u32 sc[NBINS];
  if (threadIdx.x < NBINS) sc[threadIdx.x] = 0;
  __syncthreads();
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < nv; i += (u64)gridDim.x * blockDim.x) {
    u32 v = verts[i];
    u64 deg = off[v + 1] - off[v];
    u32 b = deg <= 8 ? 0 : deg <= 16 ? 1 : deg <= 32 ? 2 : deg <= mid_max ? 3
          : deg <= wide_max ? (deg <= WIDE_SPLIT ? 4 : 6) : 5;
    bin[i] = b;
    idx[i] = (u32)i;
    atomicAdd(&sc[b], 1u);
    if (b == 5) atomicMax(maxdeg, (unsigned long long)deg);
  }
  __syncthreads();
  if (threadIdx.x < NBINS && sc[threadIdx.x]) atomicAdd(&counts[threadIdx.x], sc[threadIdx.x]);
}

// Sort keys that order vertices by degree, largest first.
__global__ void k_degree_keys(const u32* verts, const u32* idx, u32 nb, const u64* off, u32* key) {
  for (u64 t = blockIdx.x * (u64)blockDim.x + threadIdx.x; t < nb; t += (u64)gridDim.x * blockDim.x) {
    const u32 v = verts[idx[t]];
    const u64 deg = off[v + 1] - off[v];
    key[t] = 0xFFFFFFFFu - (u32)(deg < 0xFFFFFFFFull ? deg : 0xFFFFFFFFull);
  }
}

__global__ void k_fill_u32(u32* p, u32 v, u64 n) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    p[i] = v;
}

static size_t big_smem() {
  return (size_t)BIG_TAB * (8 + 4 + 4) + (size_t)BIG_THREADS * (8 + 4 + 4) +
         (size_t)BIG_LIST * sizeof(unsigned short);
}

static std::atomic<bool> g_big_attr_set[64];

constexpr u32 WIDE_MAX_BLOCKS = 148u * 3u;        // resident blocks of the full-size wide kernel
constexpr u32 WIDE_SPLIT_MAX_BLOCKS = 148u * 5u;  // and of the half-size one
constexpr u32 BIG_MAX_BLOCKS = 148u * 3u;
constexpr u32 OVF_BLOCKS = 32;  // least blocks (global regions) for rows deferred by pass 1
constexpr u64 OVF_TABLE_BYTES = 4ull << 30;  // table bytes pass 2 may spread over its blocks

// The partitioned second pass over the rows pass 1 deferred (integral
// weights).  Rows are taken in rounds whose entries fit PB_ROUND_ENTRIES;
// rows with an overflowing bucket are returned in S.pb_fail (count in
// S.pb_failcnt[0]) for the global-table pass.  Returns that count.
constexpr u64 PB_ROUND_ENTRIES = 96ull << 20;

// Entries per round of the partitioned pass forced by hl_dbg_set_pb_round
// (0: PB_ROUND_ENTRIES).
std::atomic<u64> g_dbg_pb_round{0};

template <int KIND>
static u32 huge_partitioned(Engine& E, const EvalArgs& a) {
  Scratch& S = E.sc;
  cudaStream_t st = E.stream;
  cudaEvent_t ev = E.kt_begin();
  const u32 m = E.read_u32(S.ovf_cnt.p);
  if (!m) {
    E.kt_end(KT_EVAL_PB, ev);
    return 0;
  }
  S.pb_nb.ensure(E.mem, m);
  S.pb_nc.ensure(E.mem, m);
  S.pb_bbase.ensure(E.mem, m);
  S.pb_cbase.ensure(E.mem, m);
  S.pb_ne.ensure(E.mem, m);
  S.pb_ebase.ensure(E.mem, m);
  S.pb_wcur.ensure(E.mem, m);
  S.pb_rowfail.ensure(E.mem, m);
  S.pb_fail.ensure(E.mem, m);
  S.pb_failcnt.ensure(E.mem, 2);
  ++E.nlaunch, k_pb_plan<<<grid_for(m), 256, 0, st>>>(S.ovf.p, S.ovf_cnt.p, a.verts, a.off,
                                                       S.pb_nb.p, S.pb_ne.p, S.pb_nc.p);
  HL_LAUNCH_CHECK();
  {
    u32* x = S.pb_nb.p;
    u32* y = S.pb_bbase.p;
    cub_run(E, [&](void* t, size_t& b) { return cub::DeviceScan::ExclusiveSum(t, b, x, y, (int64_t)m, st); });
    u32* x2 = S.pb_nc.p;
    u32* y2 = S.pb_cbase.p;
    cub_run(E, [&](void* t, size_t& b) { return cub::DeviceScan::ExclusiveSum(t, b, x2, y2, (int64_t)m, st); });
    u64* x3 = S.pb_ne.p;
    u64* y3 = S.pb_ebase.p;
    cub_run(E, [&](void* t, size_t& b) { return cub::DeviceScan::ExclusiveSum(t, b, x3, y3, (int64_t)m, st); });
  }
  HL_CUDA(cudaMemsetAsync(S.pb_wcur.p, 0, sizeof(double) * m, st));
  HL_CUDA(cudaMemsetAsync(S.pb_rowfail.p, 0, sizeof(u32) * m, st));
  HL_CUDA(cudaMemsetAsync(S.pb_failcnt.p, 0, sizeof(u32) * 2, st));
  // the per-row plan on the host, to cut the rows into rounds
  std::vector<u64> ne(m), eb(m);
  std::vector<u32> nb(m), bb(m), nc(m), cb(m);
  HL_CUDA(cudaMemcpyAsync(ne.data(), S.pb_ne.p, sizeof(u64) * m, cudaMemcpyDeviceToHost, st));
  HL_CUDA(cudaMemcpyAsync(eb.data(), S.pb_ebase.p, sizeof(u64) * m, cudaMemcpyDeviceToHost, st));
  HL_CUDA(cudaMemcpyAsync(nb.data(), S.pb_nb.p, sizeof(u32) * m, cudaMemcpyDeviceToHost, st));
  HL_CUDA(cudaMemcpyAsync(bb.data(), S.pb_bbase.p, sizeof(u32) * m, cudaMemcpyDeviceToHost, st));
  HL_CUDA(cudaMemcpyAsync(nc.data(), S.pb_nc.p, sizeof(u32) * m, cudaMemcpyDeviceToHost, st));
  HL_CUDA(cudaMemcpyAsync(cb.data(), S.pb_cbase.p, sizeof(u32) * m, cudaMemcpyDeviceToHost, st));
  E.sync();
  const u32 nbk = bb[m - 1] + nb[m - 1], nch = cb[m - 1] + nc[m - 1];
  S.pb_brow.ensure(E.mem, nbk);
  S.pb_crow.ensure(E.mem, nch);
  S.pb_rv.ensure(E.mem, m);
  S.pb_rfv.ensure(E.mem, m);
  S.pb_rcur.ensure(E.mem, m);
  S.pb_rkv.ensure(E.mem, m);
  S.pb_rdcur.ensure(E.mem, m);
  S.pb_ro0.ensure(E.mem, m);
  ++E.nlaunch, k_pb_rows<KIND><<<grid_for((u64)m * 32), 256, 0, st>>>(
      a, S.ovf.p, m, S.pb_nb.p, S.pb_bbase.p, S.pb_nc.p, S.pb_cbase.p, S.pb_brow.p, S.pb_crow.p,
      S.pb_rv.p, S.pb_rfv.p, S.pb_rcur.p, S.pb_rkv.p, S.pb_rdcur.p, S.pb_ro0.p);
  HL_LAUNCH_CHECK();
  PbArgs P{};
  P.ovf = S.ovf.p;
  P.nb = S.pb_nb.p;
  P.ebase = S.pb_ebase.p;
  P.bbase = S.pb_bbase.p;
  P.cbase = S.pb_cbase.p;
  P.wcur = S.pb_wcur.p;
  P.rowfail = S.pb_rowfail.p;
  P.brow = S.pb_brow.p;
  P.crow = S.pb_crow.p;
  P.rv = S.pb_rv.p;
  P.rfv = S.pb_rfv.p;
  P.rcur = S.pb_rcur.p;
  P.rkv = S.pb_rkv.p;
  P.rdcur = S.pb_rdcur.p;
  P.ro0 = S.pb_ro0.p;
  P.ne = S.pb_ne.p;
  const u64 round_entries = g_dbg_pb_round.load() ? g_dbg_pb_round.load() : PB_ROUND_ENTRIES;
  u32 r0 = 0;
  while (r0 < m) {
    u32 r1 = r0 + 1;
    while (r1 < m && eb[r1] + ne[r1] - eb[r0] <= round_entries) ++r1;
    const u64 te = eb[r1 - 1] + ne[r1 - 1] - eb[r0];
    // adjacency entries through the pass (16 algorithmic bytes each: col, w,
    // the neighbour's label)
    E.kagg[KT_EVAL_PB].items += te;
    E.kagg[KT_EVAL_PB].bytes += 16 * te;
    const u32 tb = bb[r1 - 1] + nb[r1 - 1] - bb[r0];
    S.pb_ktmp.ensure(E.mem, te);
    S.pb_ekey.ensure(E.mem, te);
    S.pb_epos.ensure(E.mem, te);
    S.pb_ew.ensure(E.mem, te);
    S.pb_bcnt.ensure(E.mem, (size_t)tb + 1);
    S.pb_boff.ensure(E.mem, (size_t)tb + 1);
    S.pb_bg.ensure(E.mem, tb);
    S.pb_bp.ensure(E.mem, tb);
    S.pb_bk.ensure(E.mem, tb);
    P.ktmp = S.pb_ktmp.p;
    P.bcnt = S.pb_bcnt.p;
    P.boff = S.pb_boff.p;
    P.ekey = S.pb_ekey.p;
    P.epos = S.pb_epos.p;
    P.ew = S.pb_ew.p;
    P.bg = S.pb_bg.p;
    P.bp = S.pb_bp.p;
    P.bk = S.pb_bk.p;
    P.r0 = r0;
    P.r1 = r1;
    P.e0 = eb[r0];
    P.b0 = bb[r0];
    P.c0 = cb[r0];
    P.c1 = cb[r1 - 1] + nc[r1 - 1];
    const u32 nchunks = P.c1 - P.c0;
    const u32 cgrid = nchunks < 148u * 8u ? nchunks : 148u * 8u;
    HL_CUDA(cudaMemsetAsync(S.pb_bcnt.p, 0, sizeof(u32) * ((size_t)tb + 1), st));
    ++E.nlaunch, k_pb_hist<KIND><<<cgrid, 256, 0, st>>>(a, P);
    HL_LAUNCH_CHECK();
    {
      u32* x = S.pb_bcnt.p;
      u32* y = S.pb_boff.p;
      cub_run(E, [&](void* t, size_t& b) {
        return cub::DeviceScan::ExclusiveSum(t, b, x, y, (int64_t)tb + 1, st);
      });
    }
    HL_CUDA(cudaMemsetAsync(S.pb_bcnt.p, 0, sizeof(u32) * ((size_t)tb + 1), st));
    ++E.nlaunch, k_pb_scatter<<<cgrid, 256, 0, st>>>(a, P);
    // fold order: buckets by entry count, largest first
    S.pb_okey.ensure(E.mem, tb);
    S.pb_okey2.ensure(E.mem, tb);
    S.pb_oval.ensure(E.mem, tb);
    S.pb_ord.ensure(E.mem, tb);
    S.pb_fwork.ensure(E.mem, 1);
    ++E.nlaunch, k_pb_order_keys<<<grid_for(tb), 256, 0, st>>>(S.pb_boff.p, tb, S.pb_okey.p,
                                                                S.pb_oval.p);
    {
      u32* ki = S.pb_okey.p;
      u32* ko = S.pb_okey2.p;
      u32* vi = S.pb_oval.p;
      u32* vo = S.pb_ord.p;
      const int kb = bits_for(te);
      cub_run(E, [&](void* t, size_t& b) {
        return cub::DeviceRadixSort::SortPairsDescending(t, b, ki, ko, vi, vo, (int64_t)tb, 0,
                                                         kb, st);
      });
    }
    HL_CUDA(cudaMemsetAsync(S.pb_fwork.p, 0, sizeof(u32), st));
    P.border = S.pb_ord.p;
    P.fold_work = S.pb_fwork.p;
    const u32 fblocks = (tb + PB_FOLD_WARPS - 1) / PB_FOLD_WARPS;
    const u32 fgrid = fblocks < 148u * 6u ? fblocks : 148u * 6u;
    u32 lim = g_pb_slots.load();
    if (lim < 64 || lim > PB_TAB) lim = PB_TAB;
    ++E.nlaunch, k_pb_fold<KIND><<<fgrid, PB_FOLD_WARPS * 32, PB_FOLD_SMEM, st>>>(a, P, tb, lim);
    ++E.nlaunch, k_pb_final<KIND><<<grid_for((u64)(r1 - r0) * 32), 256, 0, st>>>(
        a, P, S.pb_fail.p, S.pb_failcnt.p);
    HL_LAUNCH_CHECK();
    r0 = r1;
  }
  const u32 nfail = E.read_u32(S.pb_failcnt.p);
  E.kt_end(KT_EVAL_PB, ev);
  return nfail;
}

void run_eval(Engine& E, int kind, const u32* verts, u32 nv, const Level& L, const u32* s,
              const double* d, const u8* blocked, bool allow_empty, u32* out_to, double* out_gain,
              unsigned long long* counters) {
  if (!nv) return;
  cudaStream_t st = E.stream;
  Scratch& S = E.sc;
  S.order.ensure(E.mem, nv);
  S.order2.ensure(E.mem, nv);
  S.used.ensure(E.mem, nv);
  S.rank.ensure(E.mem, nv);
  S.cnt.ensure(E.mem, 16);
  u32* cnt = S.cnt.p + 2;  // NBINS bin counters (cnt[2..8])
  HL_CUDA(cudaMemsetAsync(cnt, 0, NBINS * sizeof(u32), st));
  // [0] deferred rows, [2..3] largest degree of the block bin, [4..5] work
  // counters of the block kernel's two passes
  S.ovf_cnt.ensure(E.mem, 6);
  unsigned long long* maxdeg = reinterpret_cast<unsigned long long*>(S.ovf_cnt.p + 2);
  HL_CUDA(cudaMemsetAsync(S.ovf_cnt.p, 0, 6 * sizeof(u32), st));
  // degree thresholds of the warp bins (autotuned per handle, within the
  // compile-time table sizes: mid <= MID_MAX, wide <= WIDE_MAX)
  const u32 mid_max = E.tune.mid_max ? E.tune.mid_max : MID_MAX;
  const u32 wide_max = E.tune.wide_max ? E.tune.wide_max : WIDE_MAX;
  ++E.nlaunch, k_bin<<<grid_for(nv), 256, 0, st>>>(verts, nv, L.g.off.p, S.used.p, S.order.p, cnt,
                                                    maxdeg, mid_max, wide_max);
  HL_LAUNCH_CHECK();
  u32* ki = S.used.p;
  u32* ko = S.rank.p;
  u32* vi = S.order.p;
  u32* vo = S.order2.p;
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceRadixSort::SortPairs(t, b, ki, ko, vi, vo, (int64_t)nv, 0, 3, st);
  });
  u32 c[NBINS];
  static_assert(NBINS * sizeof(u32) <= 4 * sizeof(u64), "bin counts fit before the degree");
  HL_CUDA(cudaMemcpyAsync(E.hs.p, cnt, NBINS * sizeof(u32), cudaMemcpyDeviceToHost, st));
  HL_CUDA(cudaMemcpyAsync(E.hs.p + 4, maxdeg, sizeof(u64), cudaMemcpyDeviceToHost, st));
  E.sync();
  std::memcpy(c, E.hs.p, sizeof(c));
  const u64 big_maxdeg = E.hs.p[4];
  u32 start[NBINS + 1] = {0};
  for (int b = 0; b < NBINS; ++b) start[b + 1] = start[b] + c[b];

  int dev = E.device;
  if (dev >= 0 && dev < 64 && !g_big_attr_set[dev]) {
    HL_CUDA(cudaFuncSetAttribute(k_eval_big<EVAL_MOVE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)big_smem()));
    HL_CUDA(cudaFuncSetAttribute(k_eval_big<EVAL_REFINE>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)big_smem()));
    HL_CUDA(cudaFuncSetAttribute(k_eval_wide<EVAL_MOVE, 2 * WIDE_SPLIT>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(WideSmem<2 * WIDE_SPLIT>)));
    HL_CUDA(cudaFuncSetAttribute(k_eval_wide<EVAL_REFINE, 2 * WIDE_SPLIT>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(WideSmem<2 * WIDE_SPLIT>)));
    HL_CUDA(cudaFuncSetAttribute(k_eval_wide<EVAL_MOVE, 2 * WIDE_MAX>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(WideSmem<2 * WIDE_MAX>)));
    HL_CUDA(cudaFuncSetAttribute(k_eval_wide<EVAL_REFINE, 2 * WIDE_MAX>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(WideSmem<2 * WIDE_MAX>)));
    HL_CUDA(cudaFuncSetAttribute(k_pb_fold<EVAL_MOVE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)PB_FOLD_SMEM));
    HL_CUDA(cudaFuncSetAttribute(k_pb_fold<EVAL_REFINE>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PB_FOLD_SMEM));
    g_big_attr_set[dev] = true;
  }

  EvalArgs A;
  A.verts = verts;
  A.off = L.g.off.p;
  A.col = L.g.col.p;
  A.w = L.g.w.p;
  A.f = L.f.p;
  A.s = s;
  A.d = d;
  A.kdeg = L.k.p;
  A.blocked = blocked;
  A.tw = L.tw;
  A.gamma = E.cfg.resolution;
  A.n = L.g.n;
  A.allow_empty = allow_empty;
  A.concurrent = E.integral;
  A.out_to = out_to;
  A.out_gain = out_gain;
  A.tkey = nullptr;
  A.tpos = nullptr;
  A.tval = nullptr;
  A.tlist = nullptr;
  A.region = 0;
  A.ovf_list = nullptr;
  A.ovf_count = nullptr;
  A.nidx_dev = nullptr;
  A.work = nullptr;
  {
    const u32 dbg = g_dbg_hub_defer.load();
    const u64 tuned = E.tune.hub_defer ? E.tune.hub_defer : BIG_DIRECT_DEFER;
    A.defer_deg = E.integral ? (dbg ? dbg : tuned) : 0;
  }

  cudaEvent_t ev = E.kt_begin();
  cudaEvent_t e_s = E.kt_begin();
  for (int b = 0; b < 3; ++b) {
    if (!c[b]) continue;
    EvalArgs a = A;
    a.counters = counters;
    a.idx = vo + start[b];
    a.nidx = c[b];
    u32 G = b == 0 ? 8 : b == 1 ? 16 : 32;
    u32 blocks = grid_for((u64)c[b] * G, 256);
    if (kind == EVAL_MOVE) {
      if (G == 8) ++E.nlaunch, k_eval_small<EVAL_MOVE, 8><<<blocks, 256, 0, st>>>(a);
      else if (G == 16) ++E.nlaunch, k_eval_small<EVAL_MOVE, 16><<<blocks, 256, 0, st>>>(a);
      else ++E.nlaunch, k_eval_small<EVAL_MOVE, 32><<<blocks, 256, 0, st>>>(a);
    } else {
      if (G == 8) ++E.nlaunch, k_eval_small<EVAL_REFINE, 8><<<blocks, 256, 0, st>>>(a);
      else if (G == 16) ++E.nlaunch, k_eval_small<EVAL_REFINE, 16><<<blocks, 256, 0, st>>>(a);
      else ++E.nlaunch, k_eval_small<EVAL_REFINE, 32><<<blocks, 256, 0, st>>>(a);
    }
  }
  HL_LAUNCH_CHECK();
  E.kt_end(KT_EVAL_SMALL, e_s);
  E.kagg[KT_EVAL_SMALL].items += (u64)c[0] + c[1] + c[2];
  E.kagg[KT_EVAL_MID].items += c[3];
  E.kagg[KT_EVAL_BIG].items += (u64)c[4] + c[6];
  E.kagg[KT_EVAL_HUGE].items += c[5];
  cudaEvent_t e_m = E.kt_begin();
  if (c[3]) {
    EvalArgs a = A;
    a.counters = counters ? counters + 2 : nullptr;
    a.idx = vo + start[3];
    a.nidx = c[3];
    u32 blocks = grid_for((u64)c[3] * 32, MID_WARPS * 32);
    if (kind == EVAL_MOVE)
      ++E.nlaunch, k_eval_mid<EVAL_MOVE><<<blocks, MID_WARPS * 32, 0, st>>>(a);
    else
      ++E.nlaunch, k_eval_mid<EVAL_REFINE><<<blocks, MID_WARPS * 32, 0, st>>>(a);
  }
  HL_LAUNCH_CHECK();
  E.kt_end(KT_EVAL_MID, e_m);
  cudaEvent_t e_b = E.kt_begin();
  if (c[4]) {
    EvalArgs a = A;
    a.counters = counters ? counters + 4 : nullptr;
    a.idx = vo + start[4];
    a.nidx = c[4];
    u32 blocks = grid_for((u64)c[4] * 32, WIDE_WARPS * 32);
    if (blocks > WIDE_SPLIT_MAX_BLOCKS) blocks = WIDE_SPLIT_MAX_BLOCKS;
    constexpr u32 T = 2 * WIDE_SPLIT;
    if (kind == EVAL_MOVE)
      ++E.nlaunch, k_eval_wide<EVAL_MOVE, T><<<blocks, WIDE_WARPS * 32, sizeof(WideSmem<T>), st>>>(a);
    else
      ++E.nlaunch, k_eval_wide<EVAL_REFINE, T><<<blocks, WIDE_WARPS * 32, sizeof(WideSmem<T>), st>>>(a);
    HL_LAUNCH_CHECK();
  }
  if (c[6]) {
    EvalArgs a = A;
    a.counters = counters ? counters + 4 : nullptr;
    a.idx = vo + start[6];
    a.nidx = c[6];
    u32 blocks = grid_for((u64)c[6] * 32, WIDE_WARPS * 32);
    if (blocks > WIDE_MAX_BLOCKS) blocks = WIDE_MAX_BLOCKS;
    constexpr u32 T = 2 * WIDE_MAX;
    if (kind == EVAL_MOVE)
      ++E.nlaunch, k_eval_wide<EVAL_MOVE, T><<<blocks, WIDE_WARPS * 32, sizeof(WideSmem<T>), st>>>(a);
    else
      ++E.nlaunch, k_eval_wide<EVAL_REFINE, T><<<blocks, WIDE_WARPS * 32, sizeof(WideSmem<T>), st>>>(a);
    HL_LAUNCH_CHECK();
  }
  E.kt_end(KT_EVAL_BIG, e_b);
  cudaEvent_t e_h = E.kt_begin();
  if (c[5]) {
    // Pass 1: shared tables only; rows with more than BIG_TAB / 2 distinct keys
    // are deferred to an overflow list.
    EvalArgs a = A;
    a.counters = counters ? counters + 6 : nullptr;
    // the bin's list by degree, largest first
    S.hubk.ensure(E.mem, c[5]);
    S.hubk2.ensure(E.mem, c[5]);
    S.hubv.ensure(E.mem, c[5]);
    ++E.nlaunch, k_degree_keys<<<grid_for(c[5]), 256, 0, st>>>(verts, vo + start[5], c[5],
                                                                L.g.off.p, S.hubk.p);
    HL_LAUNCH_CHECK();
    {
      u32* ki = S.hubk.p;
      u32* ko = S.hubk2.p;
      const u32* vi = vo + start[5];
      u32* vv = S.hubv.p;
      cub_run(E, [&](void* t, size_t& b) {
        return cub::DeviceRadixSort::SortPairs(t, b, ki, ko, vi, vv, (int64_t)c[5], 0, 32, st);
      });
    }
    a.idx = S.hubv.p;
    a.nidx = c[5];
    a.work = S.ovf_cnt.p + 4;
    S.ovf.ensure(E.mem, c[5]);
    a.ovf_list = S.ovf.p;
    a.ovf_count = S.ovf_cnt.p;  // zeroed with the bin counters
    u32 blocks = c[5] < BIG_MAX_BLOCKS ? c[5] : BIG_MAX_BLOCKS;
    if (kind == EVAL_MOVE)
      ++E.nlaunch, k_eval_big<EVAL_MOVE><<<blocks, BIG_THREADS, big_smem(), st>>>(a);
    else
      ++E.nlaunch, k_eval_big<EVAL_REFINE><<<blocks, BIG_THREADS, big_smem(), st>>>(a);
    HL_LAUNCH_CHECK();
    const u32* pass2_list = S.ovf.p;
    const u32* pass2_count = S.ovf_cnt.p;
    bool pass2 = big_maxdeg > BIG_TAB / 2;
    if (pass2 && E.integral) {
      // Integral weights: the deferred rows go through the partitioned pass;
      // only rows with an overflowing bucket are left for the global tables.
      const u32 nfail = kind == EVAL_MOVE ? huge_partitioned<EVAL_MOVE>(E, a)
                                          : huge_partitioned<EVAL_REFINE>(E, a);
      pass2 = nfail != 0;
      pass2_list = S.pb_fail.p;
      pass2_count = S.pb_failcnt.p;
    }
    if (pass2) {
      // Pass 2: the deferred rows (their number is read on the device), on as
      // many blocks as OVF_TABLE_BYTES of global regions allow, each region
      // sized for the largest row of the bin.
      u64 region = 64;
      while (region < 2 * big_maxdeg) region <<= 1;
      u64 fit = OVF_TABLE_BYTES / (region * 18);
      if (fit < OVF_BLOCKS) fit = OVF_BLOCKS;
      if (fit > BIG_MAX_BLOCKS) fit = BIG_MAX_BLOCKS;
      const u32 pb = (u32)fit;
      const size_t need = (size_t)pb * region;
      if (S.huge_key.cap < need) {
        S.huge_key.ensure(E.mem, need);
        S.huge_pos.ensure(E.mem, need);
        S.huge_val.ensure(E.mem, need);
        S.huge_list.ensure(E.mem, need / 2 + 1);
        ++E.nlaunch, k_fill_u32<<<grid_for(S.huge_key.cap), 256, 0, st>>>(S.huge_key.p, NONE32,
                                                                           S.huge_key.cap);
        ++E.nlaunch, k_fill_u32<<<grid_for(S.huge_pos.cap), 256, 0, st>>>(S.huge_pos.p, NONE32,
                                                                           S.huge_pos.cap);
        HL_CUDA(cudaMemsetAsync(S.huge_val.p, 0, sizeof(double) * S.huge_val.cap, st));
        HL_LAUNCH_CHECK();
      }
      EvalArgs a2 = a;
      a2.idx = pass2_list;
      a2.nidx = 0;
      a2.nidx_dev = pass2_count;
      a2.tkey = S.huge_key.p;
      a2.tpos = S.huge_pos.p;
      a2.tval = S.huge_val.p;
      a2.tlist = S.huge_list.p;
      a2.region = region;
      a2.work = S.ovf_cnt.p + 5;
      if (kind == EVAL_MOVE)
        ++E.nlaunch, k_eval_big<EVAL_MOVE><<<pb, BIG_THREADS, big_smem(), st>>>(a2);
      else
        ++E.nlaunch, k_eval_big<EVAL_REFINE><<<pb, BIG_THREADS, big_smem(), st>>>(a2);
      HL_LAUNCH_CHECK();
    }
  }
  E.kt_end(KT_EVAL_HUGE, e_h);
  E.kt_end(kind == EVAL_MOVE ? KT_MOVE_EVAL : KT_REFINE_EVAL, ev);
}

// Autotuner of the degree bins: the evaluation of one frontier is run with
// each candidate pair of warp-bin thresholds (every pair gives the same
// results; only the split between the sub-warp, warp and block kernels
// changes) and the fastest pair is kept for the handle.  With integral
// weights the bound above which hub rows skip the block kernel's shared
// tables for the partitioned pass is then tuned the same way.  Runs once, on
// the first movement round whose frontier has at least AUTOTUNE_MIN vertices.
constexpr u32 AUTOTUNE_MIN = 20000;
constexpr u32 HUB_DEFER_CAND[] = {1, 2048, 8192, 32768};  // 1: every hub row

void autotune_bins(Engine& E, const u32* verts, u32 nv, const Level& L, const u32* s,
                   const double* d, u32* out_to, double* out_gain) {
  if (E.tune.done || nv < AUTOTUNE_MIN || (E.cfg.flags & HL_FLAG_NO_AUTOTUNE)) return;
  static const u32 cand[][2] = {{128, 512}, {64, 512}, {128, 256}, {64, 256}, {96, 384}};
  cudaEvent_t a, b;
  HL_CUDA(cudaEventCreate(&a));
  HL_CUDA(cudaEventCreate(&b));
  const bool kt = E.ktiming;
  E.ktiming = false;  // the trial runs stay out of the kernel statistics
  float best = 0.f;
  u32 bm = MID_MAX, bw = WIDE_MAX;
  for (int rep = 0; rep < 2; ++rep) {  // the first pass warms the caches and allocations
    for (const auto& c : cand) {
      E.tune.mid_max = c[0];
      E.tune.wide_max = c[1];
      HL_CUDA(cudaEventRecord(a, E.stream));
      run_eval(E, EVAL_MOVE, verts, nv, L, s, d, nullptr, true, out_to, out_gain, nullptr);
      HL_CUDA(cudaEventRecord(b, E.stream));
      HL_CUDA(cudaEventSynchronize(b));
      float ms = 0.f;
      HL_CUDA(cudaEventElapsedTime(&ms, a, b));
      if (rep == 1 && (best == 0.f || ms < best)) {
        best = ms;
        bm = c[0];
        bw = c[1];
      }
    }
  }
  E.tune.mid_max = bm;
  E.tune.wide_max = bw;
  u32 bd = 0;
  if (E.integral) {
    float bdt = 0.f;
    for (int rep = 0; rep < 2; ++rep) {
      for (u32 c : HUB_DEFER_CAND) {
        E.tune.hub_defer = c;
        HL_CUDA(cudaEventRecord(a, E.stream));
        run_eval(E, EVAL_MOVE, verts, nv, L, s, d, nullptr, true, out_to, out_gain, nullptr);
        HL_CUDA(cudaEventRecord(b, E.stream));
        HL_CUDA(cudaEventSynchronize(b));
        float ms = 0.f;
        HL_CUDA(cudaEventElapsedTime(&ms, a, b));
        if (rep == 1 && (bdt == 0.f || ms < bdt)) {
          bdt = ms;
          bd = c;
        }
      }
    }
    best = bdt;
  }
  E.ktiming = kt;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  E.tune.hub_defer = bd;
  E.tune.done = true;
  E.tune.frontier = nv;
  E.tune.best_ms = best;
}

}  // namespace hl
