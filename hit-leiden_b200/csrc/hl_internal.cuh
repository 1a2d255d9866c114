// hl_internal.cuh — shared definitions of the B200 HIT-Leiden library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/hl.h"

namespace hl {

using u8 = uint8_t;
using u32 = uint32_t;
using u64 = uint64_t;

constexpr u32 NONE32 = 0xFFFFFFFFu;

// ---------------------------------------------------------------------------
// Errors: internal code throws hl::Error; the C ABI converts it to a status and
// a thread-local message.  Nothing propagates across the boundary.
// ---------------------------------------------------------------------------
struct Error : std::runtime_error {
  hl_status status;
  Error(hl_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define HL_CUDA(call)                                                                      \
  do {                                                                                     \
    cudaError_t _e = (call);                                                               \
    if (_e != cudaSuccess) {                                                               \
      if (_e == cudaErrorMemoryAllocation)                                                 \
        throw ::hl::Error(HL_ERR_OUT_OF_MEMORY, std::string(#call ": ") +                   \
                                                    cudaGetErrorString(_e));               \
      throw ::hl::Error(HL_ERR_CUDA, std::string(__FILE__) + ":" + std::to_string(__LINE__) + \
                                         " " #call ": " + cudaGetErrorString(_e));         \
    }                                                                                      \
  } while (0)

#define HL_LAUNCH_CHECK() HL_CUDA(cudaGetLastError())

inline void require(bool ok, const std::string& msg) {
  if (!ok) throw Error(HL_ERR_INVALID_INPUT, msg);
}

// ---------------------------------------------------------------------------
// Device memory: stream-ordered allocations charged against a per-handle HBM
// budget.  Buffers only grow (geometric), so steady-state batches allocate
// nothing.
// ---------------------------------------------------------------------------
struct MemCtx {
  cudaStream_t stream = nullptr;
  u64 used = 0;
  u64 peak = 0;
  u64 budget = 0;  // 0 = unlimited
};

template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t cap = 0;
  MemCtx* ctx = nullptr;

  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), cap(o.cap), ctx(o.ctx) {
    o.p = nullptr;
    o.cap = 0;
  }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      cap = o.cap;
      ctx = o.ctx;
      o.p = nullptr;
      o.cap = 0;
    }
    return *this;
  }
  ~DBuf() { release(); }

  void release() {
    if (p && ctx) {
      cudaFreeAsync(p, ctx->stream);
      ctx->used -= cap * sizeof(T);
    }
    p = nullptr;
    cap = 0;
  }

  // Ensure capacity for n elements.  Contents are NOT preserved unless keep.
  void ensure(MemCtx& c, size_t n, bool keep = false) {
    ctx = &c;
    if (n <= cap) return;
    // a first allocation is the request plus a small fixed pad; a buffer that
    // has to grow again grows by at least half, so repeated growth stays
    // amortised
    size_t ncap = n + 256;
    if (cap && ncap < cap + cap / 2) ncap = cap + cap / 2;
    u64 bytes = (u64)ncap * sizeof(T);
    if (c.budget && c.used - (u64)cap * sizeof(T) + bytes > c.budget)
      throw Error(HL_ERR_OUT_OF_MEMORY, "HBM budget exceeded (" + std::to_string(c.used + bytes) +
                                            " > " + std::to_string(c.budget) + " bytes)");
    T* np = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&np, bytes, c.stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      size_t fr = 0, tot = 0;
      cudaMemGetInfo(&fr, &tot);
      throw Error(HL_ERR_OUT_OF_MEMORY,
                  std::string("device allocation of ") + std::to_string(bytes) +
                      " bytes failed: " + cudaGetErrorString(e) + " (this handle holds " +
                      std::to_string(c.used) + " bytes; device free " + std::to_string(fr) +
                      " of " + std::to_string(tot) + ")");
    }
    if (keep && p && cap) HL_CUDA(cudaMemcpyAsync(np, p, cap * sizeof(T), cudaMemcpyDeviceToDevice, c.stream));
    if (p) {
      cudaFreeAsync(p, c.stream);
      c.used -= (u64)cap * sizeof(T);
    }
    p = np;
    cap = ncap;
    c.used += bytes;
    if (c.used > c.peak) c.peak = c.used;
  }
  void swap(DBuf& o) {
    std::swap(p, o.p);
    std::swap(cap, o.cap);
    std::swap(ctx, o.ctx);
  }
  T* get() const { return p; }
};

// Pinned host staging for small scalar read-backs.
struct HostScalars {
  u64* p = nullptr;
  explicit HostScalars() { HL_CUDA(cudaMallocHost((void**)&p, 64 * sizeof(u64))); }
  ~HostScalars() {
    if (p) cudaFreeHost(p);
  }
};

inline u32 div_up(u64 a, u64 b) { return (u32)((a + b - 1) / b); }

// Bits that hold every value in [0, maxval] (at least 1): radix sorts of keys
// with a known bound sort only those bits.
inline int bits_for(u64 maxval) {
  int b = 1;
  while (b < 64 && (maxval >> b) != 0) ++b;
  return b;
}

// ---------------------------------------------------------------------------
// FP64 arithmetic that rounds exactly like the reference's Rust expressions.
// The library is compiled with -fmad=false; the explicit _rn intrinsics make
// the evaluation order of every gain formula visible here as well.
// ---------------------------------------------------------------------------
// ΔQ(v: C→C', γ) = (w_to - w_cur)/2m + γ·k_v·(d_cur - k_v - d_to)/(2m)²
// (parallel_frontier.rs:185-190; hit_leiden.rs:1135-1140, :1488-1495).
__device__ __forceinline__ double move_gain(double w_to, double w_cur, double tw, double gamma,
                                            double kv, double d_cur, double d_to) {
  double a = __ddiv_rn(__dsub_rn(w_to, w_cur), tw);
  double b = __dmul_rn(__dmul_rn(gamma, kv), __dsub_rn(__dsub_rn(d_cur, kv), d_to));
  return __dadd_rn(a, __ddiv_rn(b, __dmul_rn(tw, tw)));
}
// Division-free screening of one vertex's candidates before move_gain.
//
// With x = fl(w_to - w_cur), b = fl(fl(γ·k_v)·fl(fl(d_cur - k_v) - d_to)) and
// c = fl(2m·2m) computed exactly as move_gain computes them, the gain is
// g = fl(fl(x/2m) + fl(b/c)) while R = x/2m + b/c is its real value, so
// |g - R| <= 2.01u·(|x|/2m + |b|/c) (u = 2^-53: three roundings).  The proxy
// Q = fl(fl(x·c) + fl(b·2m)) equals R·2m·c up to 2.01u·T with
// T = |x·c| + |b·2m|.  If a candidate R' seen before has Q' - Q > 4.02u·(T + T')
// then R' - R exceeds both gains' rounding errors and g' > g strictly: the
// candidate can neither win nor tie and needs no exact gain.  keep() tests that
// with a margin of 16u·(T + T') (and an absolute 1e-300 for subnormal terms),
// against the largest proxy seen so far; every candidate it keeps gets its
// exact move_gain and the usual comparison, so the winner and its gain bits
// are those of the unscreened scan.  Rounding is monotone, so the comparison
// fl(Q + margin) < Q' implies Q + margin < Q'.
struct GainScreen {
  double tw, c, g, dk, wcur, qmax, tmax;
  __device__ __forceinline__ void init(double w_cur, double tw_, double gamma, double kv,
                                       double d_cur) {
    tw = tw_;
    c = __dmul_rn(tw_, tw_);
    g = __dmul_rn(gamma, kv);
    dk = __dsub_rn(d_cur, kv);
    wcur = w_cur;
    qmax = -1.0 / 0.0;
    tmax = 0.0;
  }
  __device__ __forceinline__ bool keep(double w_to, double d_to) {
    const double p1 = __dmul_rn(__dsub_rn(w_to, wcur), c);
    const double p2 = __dmul_rn(__dmul_rn(g, __dsub_rn(dk, d_to)), tw);
    const double q = __dadd_rn(p1, p2);
    const double t = __dadd_rn(fabs(p1), fabs(p2));
    const double margin = __dadd_rn(__dmul_rn(1.7763568394002505e-15, __dadd_rn(t, tmax)), 1e-300);
    if (__dadd_rn(q, margin) < qmax) return false;  // 1.776e-15 = 16u
    if (q > qmax) {
      qmax = q;
      tmax = t;
    }
    return true;
  }
};

// Gain of moving to the empty community (parallel_frontier.rs:207-211).
__device__ __forceinline__ double empty_gain(double w_cur, double tw, double gamma, double kv,
                                             double d_cur) {
  double a = __ddiv_rn(-w_cur, tw);
  double b = __dmul_rn(__dmul_rn(gamma, kv), __dsub_rn(d_cur, kv));
  return __dadd_rn(a, __ddiv_rn(b, __dmul_rn(tw, tw)));
}
// ΔQ(S→∅) of the T-filter (hit_leiden.rs:1545-1547, :1627-1629).
__device__ __forceinline__ double remove_gain(double w_sc, double tw, double gamma, double ds,
                                              double dpar) {
  double a = __ddiv_rn(-w_sc, tw);
  double b = __dmul_rn(__dmul_rn(gamma, ds), __dsub_rn(dpar, ds));
  return __dadd_rn(a, __ddiv_rn(b, __dmul_rn(tw, tw)));
}

// Left-to-right sum acc + x[a] + x[a+1] + ... + x[b-1] with every addition
// rounded in that order (the reference's sequential f64 sums), computed by a
// whole warp: lanes load 32 consecutive values at once and the sum is then
// extended in lane order through shuffles.  All lanes must call it with the
// same arguments; all lanes return the same result.  `val(t)` returns the
// t-th value; `take(t)` says whether it is part of the sum.
//
// The next chunk is loaded while the current one is folded.  A chunk with
// many taken values is folded by an unrolled pass (the 32 shuffles do not
// depend on the running sum, so only the additions form the chain); a sparse
// one walks its set lanes.
template <typename V, typename P>
__device__ __forceinline__ double warp_ordered_sum(u64 a, u64 b, double acc, V val, P take) {
  const u32 lane = threadIdx.x & 31;
  if (a >= b) return acc;
  u64 t = a + lane;
  bool ok = t < b && take(t);
  double x = ok ? val(t) : 0.0;
  for (u64 base = a; base < b; base += 32) {
    const u64 tn = base + 32 + lane;
    const bool okn = tn < b && take(tn);
    const double xn = okn ? val(tn) : 0.0;
    u32 m = __ballot_sync(0xffffffffu, ok);
    if (__popc(m) > 8) {
      // all 32 values first (independent shuffles), then the dependent chain
      double y[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) y[j] = __shfl_sync(0xffffffffu, x, j);
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if ((m >> j) & 1u) acc = __dadd_rn(acc, y[j]);
    } else {
      while (m) {
        int j = __ffs(m) - 1;
        acc = __dadd_rn(acc, __shfl_sync(0xffffffffu, x, j));
        m &= m - 1;
      }
    }
    x = xn;
    ok = okn;
  }
  return acc;
}

// The same left-to-right sum as warp_ordered_sum with every value taken, the
// same bits, computed in runs instead of one addition after another.
//
// Write the running sum as |s| = M·u, u = 2^(e-52), M in [2^52, 2^53).  A term
// y with the sign of s (or a zero) is t·u.  If t is not an odd multiple of 1/2
// and M + rnd(t) <= 2^53 - 1 (rnd: nearest integer), the exact sum stays below
// 2^(e+1), so fl(s + y) has the sign of s and the magnitude (M + rnd(t))·u:
// the rounding does not depend on s.  A run of such terms therefore adds the
// exact integer prefix sums of their rnd(t).  Lane l holds the 4 consecutive
// terms 4l..4l+3 of a 128-term tile, and one warp scan of the lanes' integer
// totals gives every prefix.  A run ends before the first term that is a tie,
// has the other sign, is not finite, or would carry M past 2^53 - 1.  From
// there the terms take ordinary rounded additions to the end of that lane's
// 4 terms (to the end of the tile when the run was shorter than 32 terms) and
// a new run starts.  A sum that is zero, subnormal, below 2^-959, infinite or
// NaN also takes ordinary additions, 4 terms at a time.
//
// Worth it from a few hundred terms on: the first terms of a sum from zero
// cross a binade every few terms.
constexpr u64 RUN_FOLD_MIN = 512;

// The terms are xs[a..b), contiguous: one warp folds one long segment, so its
// own loads must be in flight well ahead.  The tiles after the current one
// are held in registers, and the one four tiles ahead is prefetched into L2.
__device__ __forceinline__ double warp_fold_runs(u64 a, u64 b, double acc,
                                                 const double* __restrict__ xs) {
  constexpr u32 PER = 4, TILE = 32 * PER;
  constexpr u64 MAXM = (1ull << 53) - 1;
  const u32 lane = threadIdx.x & 31;
  if (a >= b) return acc;
  double x[PER], xn[PER], xnn[PER];
  auto load = [&](u64 base, double* dst) {
#pragma unroll
    for (u32 j = 0; j < PER; ++j) {
      const u64 t = base + PER * lane + j;
      dst[j] = t < b ? xs[t] : 0.0;
    }
  };
  load(a, x);
  load(a + TILE, xn);
  for (u64 base = a; base < b; base += TILE) {
    load(base + 2 * TILE, xnn);
    {
      const u64 t = base + 4 * TILE + PER * lane;
      if (t < b) asm volatile("prefetch.global.L2 [%0];" ::"l"(xs + t));
    }
    const u32 cnt = (u32)(b - base < TILE ? b - base : TILE);
    u32 q0 = 0;
    while (q0 < cnt) {
      const u64 bits = (u64)__double_as_longlong(acc);
      const u32 bexp = (u32)(bits >> 52) & 0x7ffu;
      u32 q = q0, e;
      if (bexp >= 64 && bexp <= 2046) {
        const bool neg = acc < 0.0;
        // 1/u = 2^(52-e), a normal power of two for these exponents
        const double scale = __longlong_as_double((long long)((u64)(2098u - bexp) << 52));
        const u64 M = (bits & ((1ull << 52) - 1)) | (1ull << 52);
        u64 C[PER];
        u32 badm = 0;  // bit j: this lane's term j ends the run
        u64 P = 0;
#pragma unroll
        for (u32 j = 0; j < PER; ++j) {
          const u32 idx = PER * lane + j;
          const bool in = idx >= q0 && idx < cnt;
          const double y = neg ? -x[j] : x[j];
          const double t = __dmul_rn(y, scale);  // exact, or below 2^-1022 where rnd is 0
          const bool good = (y >= 0.0) && (t < 4503599627370496.0);  // 2^52; false for NaN
          const double tg = good ? t : 0.0;
          const double f = floor(tg);
          const double fr = __dsub_rn(tg, f);  // exact
          const bool tie = fr == 0.5;
          P += (in && good && !tie) ? (u64)f + (fr > 0.5 ? 1ull : 0ull) : 0ull;
          C[j] = P;
          if (in && (!good || tie)) badm |= 1u << j;
        }
        u64 inc = P;
#pragma unroll
        for (u32 o = 1; o < 32; o <<= 1) {
          const u64 v = __shfl_up_sync(0xffffffffu, inc, o);
          if (lane >= o) inc += v;
        }
        const u64 excl = inc - P;
#pragma unroll
        for (u32 j = 0; j < PER; ++j) {
          C[j] += excl;
          const u32 idx = PER * lane + j;
          if (idx >= q0 && idx < cnt && M + C[j] > MAXM) badm |= 1u << j;
        }
        const u32 fb = badm ? (u32)(__ffs(badm) - 1) : PER;
        const u32 ball = __ballot_sync(0xffffffffu, badm != 0);
        q = cnt;
        if (ball) {
          const u32 first = (u32)(__ffs(ball) - 1);
          q = PER * first + __shfl_sync(0xffffffffu, fb, first);
        }
        if (q > q0) {
          // the prefix through term q - 1, from the lane that holds it (a
          // masked overwrite: a select by q % 4 would index C dynamically)
          u64 mine = excl;
#pragma unroll
          for (u32 j = 0; j < PER; ++j)
            if (PER * lane + j < q) mine = C[j];
          const u64 cr = __shfl_sync(0xffffffffu, mine, (q - 1) / PER);
          acc = __longlong_as_double(
              (long long)((bits & (1ull << 63)) | ((u64)bexp << 52) | (M + cr - (1ull << 52))));
        }
        if (q >= cnt) break;
        e = (q - q0 < 32) ? cnt : min(cnt, (q / PER) * PER + PER);
      } else {
        e = min(cnt, (q0 / PER) * PER + PER);
      }
      // ordinary rounded additions of the terms [q, e)
      for (u32 l = q / PER; l * PER < e; ++l) {
#pragma unroll
        for (u32 j = 0; j < PER; ++j) {
          const double y = __shfl_sync(0xffffffffu, x[j], l);
          const u32 idx = l * PER + j;
          if (idx >= q && idx < e) acc = __dadd_rn(acc, y);
        }
      }
      q0 = e;
    }
#pragma unroll
    for (u32 j = 0; j < PER; ++j) {
      x[j] = xn[j];
      xn[j] = xnn[j];
    }
  }
  return acc;
}

// The ordered-sum kernels come in pairs.  The first, a warp per segment with
// the few registers of warp_ordered_sum, sums the segments below RUN_FOLD_MIN
// and lists the longer ones; the second folds the listed ones in runs, with
// FOLD_BLOCKS blocks of 256 threads (one wave at up to 80 registers a
// thread) and the count read on the device.
constexpr u32 FOLD_BLOCKS = 148 * 3;

// Appends segment i to the list of long segments (lane 0 of the calling warp).
__device__ __forceinline__ void fold_defer(u32* list, u32* count, u32 i) {
  if ((threadIdx.x & 31) == 0) list[atomicAdd(count, 1u)] = i;
}

// First position in [lo, hi) of the ascending array a whose value is >= x.
__device__ __forceinline__ u64 lower_bound_u32(const u32* a, u64 lo, u64 hi, u32 x) {
  while (lo < hi) {
    u64 mid = (lo + hi) >> 1;
    if (a[mid] < x)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Total order on doubles as unsigned keys (ascending).
__device__ __forceinline__ u64 double_key(double x) {
  u64 b = (u64)__double_as_longlong(x);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

}  // namespace hl
