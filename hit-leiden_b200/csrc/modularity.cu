// modularity.cu — Q = (Σ_intra w − Σ_C d(C)²/2m) / 2m (hit_leiden.rs:121-161)
// as a segmented FP64 reduction over the resident CSR, and first-seen label
// canonicalisation (hit_leiden.rs:358-376).
//
// Each undirected edge appears twice in the CSR (a self-loop twice in its own
// row), so the CSR intra sum equals the reference's 2·Σ_intra over its edge
// list and the row sums equal its node degrees.  The reference adds the Σ_C
// terms in hash order; here every partial sum is carried as a double-double
// (error-free TwoSum), so Q is the accurately rounded value and agrees with any
// faithful ordering to ~1e-15 relative.
#include "hl_engine.cuh"

namespace hl {

static inline u32 grid_for(u64 n, u32 block = 256) {
  u64 g = (n + block - 1) / block;
  if (g > 148u * 64u) g = 148u * 64u;
  return g ? (u32)g : 1u;
}

struct DD {
  double hi, lo;
};

__device__ __forceinline__ DD dd_add(DD a, double b) {
  double s = __dadd_rn(a.hi, b);
  double bb = __dsub_rn(s, a.hi);
  double err = __dadd_rn(__dsub_rn(a.hi, __dsub_rn(s, bb)), __dsub_rn(b, bb));
  return {s, __dadd_rn(a.lo, err)};
}
__device__ __forceinline__ DD dd_add(DD a, DD b) {
  DD r = dd_add(a, b.hi);
  r.lo = __dadd_rn(r.lo, b.lo);
  return r;
}

// Per-row intra weight (exact for integral weights; at most deg roundings else).
__global__ void k_row_intra(u32 n, const u64* off, const u32* col, const double* w,
                            const u32* part, double* out) {
  const u32 lane = threadIdx.x & 31;
  const u64 warp = (blockIdx.x * (u64)blockDim.x + threadIdx.x) >> 5;
  const u64 nwarps = ((u64)gridDim.x * blockDim.x) >> 5;
  for (u64 v = warp; v < n; v += nwarps) {
    u32 c = part[v];
    DD s{0.0, 0.0};
    for (u64 p = off[v] + lane; p < off[v + 1]; p += 32)
      if (part[col[p]] == c) s = dd_add(s, w[p]);
    for (int o = 16; o; o >>= 1) {
      DD t{__shfl_xor_sync(0xffffffffu, s.hi, o), __shfl_xor_sync(0xffffffffu, s.lo, o)};
      s = dd_add(s, t);
    }
    if (lane == 0) out[v] = s.hi + s.lo;
  }
}

__global__ void k_sq_terms(u32 nc, const double* d, double tw, double* out) {
  for (u64 c = blockIdx.x * (u64)blockDim.x + threadIdx.x; c < nc; c += (u64)gridDim.x * blockDim.x) {
    double x = d[c];
    out[c] = __ddiv_rn(__dmul_rn(x, x), tw);
  }
}

// Double-double block reduction → one DD per block.
__global__ void k_dd_reduce(const double* x, const double* xlo, u64 n, double* ohi, double* olo) {
  __shared__ double sh[256], sl[256];
  DD s{0.0, 0.0};
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
    s = dd_add(s, x[i]);
    if (xlo) s.lo = __dadd_rn(s.lo, xlo[i]);
  }
  sh[threadIdx.x] = s.hi;
  sl[threadIdx.x] = s.lo;
  __syncthreads();
  for (u32 st = blockDim.x / 2; st; st >>= 1) {
    if (threadIdx.x < st) {
      DD a{sh[threadIdx.x], sl[threadIdx.x]}, b{sh[threadIdx.x + st], sl[threadIdx.x + st]};
      DD r = dd_add(a, b);
      sh[threadIdx.x] = r.hi;
      sl[threadIdx.x] = r.lo;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    ohi[blockIdx.x] = sh[0];
    olo[blockIdx.x] = sl[0];
  }
}

static double dd_sum(Engine& E, const double* x, u64 n) {
  if (!n) return 0.0;
  Scratch& S = E.sc;
  u32 blocks = grid_for(n);
  if (blocks > 1024) blocks = 1024;
  S.red.ensure(E.mem, 2 * (size_t)blocks + 4);
  S.red2.ensure(E.mem, 4);
  ++E.nlaunch, k_dd_reduce<<<blocks, 256, 0, E.stream>>>(x, nullptr, n, S.red.p, S.red.p + blocks);
  ++E.nlaunch, k_dd_reduce<<<1, 256, 0, E.stream>>>(S.red.p, S.red.p + blocks, blocks, S.red2.p, S.red2.p + 1);
  HL_LAUNCH_CHECK();
  double hi = E.read_f64(S.red2.p);
  double lo = E.read_f64(S.red2.p + 1);
  return hi + lo;
}

double modularity(Engine& E, Level& L, const u32* part) {
  const u32 n = L.g.n;
  if (!n || L.tw == 0.0) return 0.0;
  Scratch& S = E.sc;
  cudaStream_t st = E.stream;
  // intra
  DBuf<double> rows;
  rows.ensure(E.mem, n);
  ++E.nlaunch, k_row_intra<<<grid_for((u64)n * 32), 256, 0, st>>>(n, L.g.off.p, L.g.col.p, L.g.w.p, part,
                                                      rows.p);
  HL_LAUNCH_CHECK();
  double intra = dd_sum(E, rows.p, n);
  // Σ_C d(C)²/2m
  S.cnt.ensure(E.mem, 16);
  u32* o = S.cnt.p + 13;
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceReduce::Max(t, b, part, o, (int64_t)n, st);
  });
  u32 nc = E.read_u32(o) + 1;
  DBuf<double> d, terms;
  d.ensure(E.mem, nc);
  terms.ensure(E.mem, nc);
  recompute_comm_degrees(E, L, part, nc, d.p);
  ++E.nlaunch, k_sq_terms<<<grid_for(nc), 256, 0, st>>>(nc, d.p, L.tw, terms.p);
  HL_LAUNCH_CHECK();
  double expected = dd_sum(E, terms.p, nc);
  return (intra - expected) / L.tw;
}

// First-seen relabelling: a label's new id is the rank of its first index.
__global__ void k_first_index(const u32* lab, u64 n, u32* first) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    atomicMin(&first[lab[i]], (u32)i);
}
__global__ void k_is_first(const u32* lab, u64 n, const u32* first, u32* flag) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    flag[i] = first[lab[i]] == (u32)i ? 1u : 0u;
}
__global__ void k_apply_first(const u32* lab, u64 n, const u32* first, const u32* rank, u32* out) {
  for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    out[i] = rank[first[lab[i]]];
}

void canonicalize_device(Engine& E, u32* labels, u64 n, u32* out) {
  if (!n) return;
  Scratch& S = E.sc;
  cudaStream_t st = E.stream;
  S.cnt.ensure(E.mem, 16);
  u32* o = S.cnt.p + 14;
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceReduce::Max(t, b, labels, o, (int64_t)n, st);
  });
  u64 nc = (u64)E.read_u32(o) + 1;
  DBuf<u32> first, flag, rank;
  first.ensure(E.mem, nc);
  flag.ensure(E.mem, n);
  rank.ensure(E.mem, n);
  HL_CUDA(cudaMemsetAsync(first.p, 0xFF, sizeof(u32) * nc, st));
  ++E.nlaunch, k_first_index<<<grid_for(n), 256, 0, st>>>(labels, n, first.p);
  ++E.nlaunch, k_is_first<<<grid_for(n), 256, 0, st>>>(labels, n, first.p, flag.p);
  HL_LAUNCH_CHECK();
  u32* a = flag.p;
  u32* r = rank.p;
  cub_run(E, [&](void* t, size_t& b) {
    return cub::DeviceScan::ExclusiveSum(t, b, a, r, (int64_t)n, st);
  });
  ++E.nlaunch, k_apply_first<<<grid_for(n), 256, 0, st>>>(labels, n, first.p, rank.p, out);
  HL_LAUNCH_CHECK();
  E.sync();
}

}  // namespace hl
