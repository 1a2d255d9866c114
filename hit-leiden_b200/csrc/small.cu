// small.cu — throughput-mode movement rounds with a small frontier, all in
// one block (hit_leiden.rs:1068-1101 → throughput.rs:80-236).
//
// Late rounds, upper levels and small graphs have a few hundred active
// vertices: there the round-by-round path is bound by its launches and by
// the host reads between them (frontier size, bin counts, candidate count,
// selection progress), not by the GPU.  This kernel runs whole rounds without
// leaving the device:
//   1. the frontier (a list; the first one from the active flags);
//   2. each active vertex's best move on the round's snapshot, a warp per
//      vertex with its table in shared memory: per-key sums in CSR order, the
//      first CSR position on ties, the empty community n + v on a strict
//      improvement — the same rules and bits as the evaluation kernels;
//   3. the positive candidates sorted by (gain desc, node asc) (bitonic);
//   4. the reference's greedy decoupled selection, in rank order;
//   5. the accepted moves applied in that order (d(C) updated in that order);
//   6. the next frontier and the K marks from the moved vertices.
// A round is atomic: the kernel hands the loop back to the host at a round
// boundary (frontier flags complete) when the next frontier would exceed
// SM_FRONTIER vertices or an active vertex has more than SM_MAXDEG entries,
// and the host continues with the multi-kernel rounds.  Nothing waits on
// another block; every loop is bounded by the round cap.
#include <cstring>

#include "hl_engine.cuh"

namespace hl {

constexpr u32 SM_THREADS = 512;
constexpr u32 SM_WARPS = SM_THREADS / 32;
constexpr u32 SM_MAXDEG = 256;     // degree limit of a warp's table
constexpr u32 SM_TAB = 2 * SM_MAXDEG;
constexpr u32 SM_FRONTIER = 4096;  // frontier (and candidate) limit; a power of two
constexpr u32 SMALL_N_MAX = 1u << 18;

enum : u32 { SM_DONE = 0, SM_BIG_FRONTIER = 1, SM_BIG_DEGREE = 2 };
enum : u32 { SM_ROLE_EMIT = 1, SM_ROLE_ACC = 2 };

struct SmallSmem {
  double tv[SM_WARPS][SM_TAB];
  u32 tk[SM_WARPS][SM_TAB];
  u32 tp[SM_WARPS][SM_TAB];
  double sw[SM_WARPS][32];
  unsigned long long skey[SM_FRONTIER];  // ~double_key(gain): ascending = gain descending
  u32 snode[SM_FRONTIER];
  u32 sidx[SM_FRONTIER];                 // frontier index of the candidate
  u32 sel[SM_FRONTIER];                  // accepted frontier indices, in rank order
};

struct SmallArgs {
  u32 n;
  const u64* off;
  const u32* col;
  const double* w;
  u32* f;
  const u32* s;
  const double* k;
  double* d;
  u8* flags_cur;   // the frontier as 0/1 bytes (S.active)
  u8* flags_nxt;   // all zero on entry (S.next)
  u8* changed;
  u8* affected;
  bool mark_moved;
  double tw, gamma;
  u32* role;       // per community: (selection round << 2) | roles
  u32 round0;      // last selection round id used before this call
  u32 it0, max_rounds;
  u32* list_a;     // frontier lists, SM_FRONTIER entries each
  u32* list_b;
  u32* cand_to;
  double* cand_gain;
  unsigned long long* out;  // see k_move_small's epilogue
};

__device__ __forceinline__ u32 sm_hash(u32 x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

__device__ __forceinline__ u32 sm_role_bits(u32 r, u32 round) {
  return (r >> 2) == round ? (r & 3u) : 0u;
}

// Best move of v (the evaluation kernels' rules), by one warp.
__device__ __forceinline__ void sm_eval_vertex(const SmallArgs& A, SmallSmem& S, u32 wib,
                                               u32 v, u32& to_out, double& gain_out) {
  const u32 lane = threadIdx.x & 31;
  const u64 o0 = A.off[v], o1 = A.off[v + 1];
  const u64 deg = o1 - o0;
  const u32 cur = A.f[v];
  const double kv = A.k[v];
  u32* tk = S.tk[wib];
  u32* tp = S.tp[wib];
  double* tv = S.tv[wib];
  u32 cap = 64;
  while (cap < 2 * deg) cap <<= 1;
  const u32 mask = cap - 1;
  for (u32 x = lane; x < cap; x += 32) tk[x] = NONE32;
  __syncwarp();
  for (u64 b0 = o0; b0 < o1; b0 += 32) {
    const u64 q = b0 + lane;
    u32 key = NONE32;
    double wv = 0.0;
    bool has = false;
    if (q < o1) {
      const u32 nb = A.col[q];
      wv = A.w[q];
      if (nb != v) {  // self-loops skipped (parallel_frontier.rs:164-166)
        key = A.f[nb];
        has = true;
      }
    }
    S.sw[wib][lane] = wv;
    __syncwarp();
    const u32 grp = __match_any_sync(0xffffffffu, key);
    if (has && lane == (u32)(__ffs(grp) - 1)) {
      u32 slot = sm_hash(key) & mask;
      while (true) {  // at most cap probes: the table holds at most deg < cap keys
        const u32 prev = atomicCAS(&tk[slot], NONE32, key);
        if (prev == NONE32 || prev == key) {
          double sum = prev == NONE32 ? 0.0 : tv[slot];
          for (u32 m = grp; m; m &= m - 1) sum = __dadd_rn(sum, S.sw[wib][__ffs(m) - 1]);
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
  const u32 fm = __ballot_sync(0xffffffffu, found);
  wcur = __shfl_sync(0xffffffffu, wcur, fm ? __ffs(fm) - 1 : 0);
  if (!fm) wcur = 0.0;
  double g = -1.0;
  u32 p = NONE32, kk = cur;
  if (A.tw != 0.0) {
    for (u32 x = lane; x < cap; x += 32) {
      const u32 key = tk[x];
      if (key == NONE32 || key == cur) continue;
      const double gn = move_gain(tv[x], wcur, A.tw, A.gamma, kv, A.d[cur], A.d[key]);
      const u32 pp = tp[x];
      if (p == NONE32 || gn > g || (gn == g && pp < p)) {
        g = gn;
        p = pp;
        kk = key;
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
  // the decision (the evaluation kernels' finish(): best neighbour community
  // on a positive gain, then the empty community on a strict improvement)
  u32 to = cur;
  double gain = 0.0;
  if (p != NONE32 && g > 0.0) {
    gain = g;
    to = kk;
  }
  if (A.tw != 0.0) {
    const double eg = empty_gain(wcur, A.tw, A.gamma, kv, A.d[cur]);
    if (eg > gain) {
      gain = eg;
      to = A.n + v;
    }
  }
  to_out = to;
  gain_out = gain;
}

__global__ void __launch_bounds__(SM_THREADS, 1) k_move_small(SmallArgs A) {
  extern __shared__ __align__(16) unsigned char sm_raw[];
  SmallSmem& S = *reinterpret_cast<SmallSmem*>(sm_raw);
  __shared__ u32 s_na, s_nn, s_m, s_nacc, s_big, s_over;
  __shared__ u32 s_wcnt[SM_WARPS];
  const u32 tid = threadIdx.x, lane = tid & 31, wib = tid >> 5;
  const u32 lt = (1u << lane) - 1u;
  unsigned long long trav = 0;
  unsigned long long moves = 0, cands = 0, sum_nv = 0;  // thread 0
  u8* fcur = A.flags_cur;
  u8* fnxt = A.flags_nxt;
  u32* lcur = A.list_a;
  u32* lnxt = A.list_b;
  u32 it = A.it0;
  u32 round = A.round0;
  u32 cur_is_next = 0;  // which flag array holds the current frontier
  // ---- the first frontier: the active flags, compacted in node order ----
  if (tid == 0) {
    s_na = 0;
    s_over = 0;
  }
  __syncthreads();
  for (u32 base = 0; base < A.n; base += SM_THREADS) {
    const u32 v = base + tid;
    const bool fl = v < A.n && fcur[v] != 0;
    const u32 b = __ballot_sync(0xffffffffu, fl);
    if (lane == 0) s_wcnt[wib] = __popc(b);
    __syncthreads();
    u32 pos = s_na;
    for (u32 x = 0; x < wib; ++x) pos += s_wcnt[x];
    pos += __popc(b & lt);
    if (fl) {
      if (pos < SM_FRONTIER) lcur[pos] = v;
      else s_over = 1;
    }
    __syncthreads();
    if (tid == 0)
      for (u32 x = 0; x < SM_WARPS; ++x) s_na += s_wcnt[x];
    __syncthreads();
    if (s_over) break;  // uniform
  }
  u32 status = SM_DONE;
  while (true) {
    if (s_over) {
      status = SM_BIG_FRONTIER;
      break;
    }
    const u32 na = s_na;
    if (it >= A.max_rounds || na == 0) break;
    // every active vertex must fit a warp table
    if (tid == 0) s_big = 0;
    __syncthreads();
    for (u32 i = tid; i < na; i += SM_THREADS) {
      const u32 v = lcur[i];
      if (A.off[v + 1] - A.off[v] > SM_MAXDEG) s_big = 1;
    }
    __syncthreads();
    if (s_big) {
      status = SM_BIG_DEGREE;
      break;
    }
    // the round runs here: the current flags are cleared for reuse as the
    // next round's target
    for (u32 i = tid; i < na; i += SM_THREADS) fcur[lcur[i]] = 0;
    if (tid == 0) sum_nv += na;
    // ---- evaluation on the snapshot ----
    for (u32 i = wib; i < na; i += SM_WARPS) {
      const u32 v = lcur[i];
      u32 to;
      double gain;
      sm_eval_vertex(A, S, wib, v, to, gain);
      if (lane == 0) {
        A.cand_to[i] = to;
        A.cand_gain[i] = gain;
        trav += A.off[v + 1] - A.off[v];
      }
    }
    __syncthreads();
    // ---- positive candidates, sorted by (gain desc, node asc) ----
    if (tid == 0) s_m = 0;
    __syncthreads();
    for (u32 i = tid; i < na; i += SM_THREADS) {
      const double gn = A.cand_gain[i];
      if (gn > 0.0) {
        const u32 slot = atomicAdd(&s_m, 1u);
        S.skey[slot] = ~double_key(gn);
        S.snode[slot] = lcur[i];
        S.sidx[slot] = i;
      }
    }
    __syncthreads();
    const u32 M = s_m;
    ++it;
    if (tid == 0) cands += M;
    if (M == 0) break;  // nothing selected: the next frontier is empty
    u32 P = 1;
    while (P < M) P <<= 1;
    for (u32 i = M + tid; i < P; i += SM_THREADS) {
      S.skey[i] = ~0ull;
      S.snode[i] = NONE32;
      S.sidx[i] = NONE32;
    }
    __syncthreads();
    for (u32 size = 2; size <= P; size <<= 1) {
      for (u32 stride = size >> 1; stride > 0; stride >>= 1) {
        for (u32 i = tid; i < P; i += SM_THREADS) {
          const u32 j = i ^ stride;
          if (j > i) {
            const bool up = (i & size) == 0;
            const unsigned long long ki = S.skey[i], kj = S.skey[j];
            const u32 ni = S.snode[i], nj = S.snode[j];
            const bool gt = ki > kj || (ki == kj && ni > nj);
            if (gt == up) {
              S.skey[i] = kj;
              S.skey[j] = ki;
              S.snode[i] = nj;
              S.snode[j] = ni;
              const u32 t = S.sidx[i];
              S.sidx[i] = S.sidx[j];
              S.sidx[j] = t;
            }
          }
        }
        __syncthreads();
      }
    }
    // ---- greedy decoupled selection and the moves, in rank order ----
    if (tid == 0) {
      ++round;
      u32 nacc = 0;
      for (u32 r = 0; r < M; ++r) {
        const u32 i = S.sidx[r];
        const u32 v = S.snode[r];
        const u32 from = A.f[v], to = A.cand_to[i];
        const u32 ba = sm_role_bits(A.role[from], round);
        const u32 bb = sm_role_bits(A.role[to], round);
        if ((ba & SM_ROLE_ACC) || (bb & SM_ROLE_EMIT)) continue;
        A.role[from] = (round << 2) | ba | SM_ROLE_EMIT;
        A.role[to] = (round << 2) | sm_role_bits(A.role[to], round) | SM_ROLE_ACC;
        S.sel[nacc++] = i;
      }
      for (u32 j = 0; j < nacc; ++j) {
        const u32 i = S.sel[j];
        const u32 v = lcur[i];
        const u32 from = A.f[v], to = A.cand_to[i];
        const double kv = A.k[v];
        A.f[v] = to;
        A.changed[v] = 1;
        if (A.mark_moved) A.affected[v] = 1;
        A.d[from] = __dsub_rn(A.d[from], kv);
        A.d[to] = __dadd_rn(A.d[to], kv);
      }
      moves += nacc;
      s_nacc = nacc;
      s_nn = 0;
      s_over = 0;
    }
    __syncthreads();
    // ---- the next frontier and K (throughput.rs:189-199), after all moves ----
    const u32 nacc = s_nacc;
    for (u32 j = wib; j < nacc; j += SM_WARPS) {
      const u32 v = lcur[S.sel[j]];
      const u32 to = A.f[v];
      const u32 sv = A.s[v];
      bool any_same = false;
      for (u64 q = A.off[v] + lane; q < A.off[v + 1]; q += 32) {
        const u32 nb = A.col[q];
        if (A.f[nb] != to) {
          // byte flag: set it once; the first setter appends nb to the list
          const u32 word = nb >> 2, sh = (nb & 3u) * 8;
          const u32 old = atomicOr(reinterpret_cast<unsigned int*>(fnxt) + word, 1u << sh);
          if (((old >> sh) & 0xFFu) == 0) {
            const u32 pos = atomicAdd(&s_nn, 1u);
            if (pos < SM_FRONTIER) lnxt[pos] = nb;
            else s_over = 1;
          }
        }
        if (A.s[nb] == sv) {
          A.affected[nb] = 1;
          any_same = true;
        }
      }
      if (__any_sync(0xffffffffu, any_same) && lane == 0) A.affected[v] = 1;
    }
    __syncthreads();
    if (tid == 0) s_na = s_nn < SM_FRONTIER ? s_nn : SM_FRONTIER;
    {
      u8* tf = fcur;
      fcur = fnxt;
      fnxt = tf;
      u32* tl = lcur;
      lcur = lnxt;
      lnxt = tl;
      cur_is_next ^= 1u;
    }
    __syncthreads();
  }
  for (int o = 16; o; o >>= 1) trav += __shfl_xor_sync(0xffffffffu, trav, o);
  __shared__ unsigned long long s_trav;
  if (tid == 0) s_trav = 0;
  __syncthreads();
  if (lane == 0 && trav) atomicAdd(&s_trav, trav);
  __syncthreads();
  if (tid == 0) {
    A.out[0] = it;
    A.out[1] = moves;
    A.out[2] = cands;
    A.out[3] = s_trav;
    A.out[4] = status;
    A.out[5] = cur_is_next;
    A.out[6] = round;
    A.out[7] = sum_nv;
  }
}

static size_t small_smem() { return sizeof(SmallSmem); }

static std::atomic<bool> g_small_attr[64];

// Runs movement rounds in one block from the current frontier (S.active).
// Returns true when the movement stage is finished; false when the host loop
// must continue (S.active then holds the next frontier).  *big_degree tells
// that a hub is active, so the caller stays on the multi-kernel rounds.
bool move_rounds_small(Engine& E, Level& L, bool mark_moved, u32& it, u64& moves, u64& cands,
                       u64& trav, u64& sum_nv, bool* big_degree) {
  *big_degree = false;
  const u32 n = L.g.n;
  if (n == 0 || n > SMALL_N_MAX) return false;
  Scratch& S = E.sc;
  cudaStream_t st = E.stream;
  const int dev = E.device;
  if (dev >= 0 && dev < 64 && !g_small_attr[dev]) {
    HL_CUDA(cudaFuncSetAttribute(k_move_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)small_smem()));
    g_small_attr[dev] = true;
  }
  S.sm_list_a.ensure(E.mem, SM_FRONTIER);
  S.sm_list_b.ensure(E.mem, SM_FRONTIER);
  S.sm_out.ensure(E.mem, 8);
  S.cand_to.ensure(E.mem, SM_FRONTIER);
  S.cand_gain.ensure(E.mem, SM_FRONTIER);
  HL_CUDA(cudaMemsetAsync(S.next.p, 0, ((size_t)n + 3) & ~(size_t)3, st));
  u32 round0 = E.sel_round;
  if (round0 + E.cfg.max_rounds + 2 >= (1u << 29)) round0 = E.sel_round = 1;
  SmallArgs A;
  A.n = n;
  A.off = L.g.off.p;
  A.col = L.g.col.p;
  A.w = L.g.w.p;
  A.f = L.f.p;
  A.s = L.s_cur.p;
  A.k = L.k.p;
  A.d = S.d.p;
  A.flags_cur = S.active.p;
  A.flags_nxt = S.next.p;
  A.changed = S.changed.p;
  A.affected = S.affected.p;
  A.mark_moved = mark_moved;
  A.tw = L.tw;
  A.gamma = E.cfg.resolution;
  A.role = S.role.p;
  A.round0 = round0;
  A.it0 = it;
  A.max_rounds = E.cfg.max_rounds ? E.cfg.max_rounds : 20;
  A.list_a = S.sm_list_a.p;
  A.list_b = S.sm_list_b.p;
  A.cand_to = S.cand_to.p;
  A.cand_gain = S.cand_gain.p;
  A.out = reinterpret_cast<unsigned long long*>(S.sm_out.p);
  cudaEvent_t ev = E.kt_begin();
  ++E.nlaunch, k_move_small<<<1, SM_THREADS, small_smem(), st>>>(A);
  HL_LAUNCH_CHECK();
  E.kt_end(KT_MOVE_SMALL, ev);
  u64 o[8];
  HL_CUDA(cudaMemcpyAsync(E.hs.p + 16, S.sm_out.p, 8 * sizeof(u64), cudaMemcpyDeviceToHost, st));
  E.sync();
  std::memcpy(o, E.hs.p + 16, sizeof(o));
  it = (u32)o[0];
  moves += o[1];
  cands += o[2];
  trav += o[3];
  sum_nv += o[7];
  E.sel_round = (u32)o[6];
  if (o[5]) S.active.swap(S.next);  // the frontier flags the loop continues from
  E.kagg[KT_MOVE_SMALL].bytes += 52ull * o[7] + 16ull * o[3] + 8ull * o[2];
  E.kagg[KT_MOVE_SMALL].items += o[7];
  if (o[4] == SM_BIG_DEGREE) *big_degree = true;
  return o[4] == SM_DONE;
}

}  // namespace hl
