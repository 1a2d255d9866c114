// hl_engine.cuh — device state of one graph handle and the stage entry points.
#pragma once
#include <atomic>
#include <initializer_list>
#include <cub/cub.cuh>

#include "hl_internal.cuh"

namespace hl {

// Undirected weighted CSR on the device: both directions stored, rows sorted
// by neighbour id, a self-loop stored twice in its row (in_memory.rs:20-72).
struct DevGraph {
  u32 n = 0;
  u64 nnz = 0;
  u64 self_loop_entries = 0;
  DBuf<u64> off;  // n+1
  DBuf<u32> col;
  DBuf<double> w;
  DBuf<u32> col2;  // the other half of the double buffer used by apply_delta
  DBuf<double> w2;
};

// One hierarchy level (state.rs:19-32): supergraph G^p and its maps.
struct Level {
  DevGraph g;
  DBuf<u32> f;      // community_mapping_per_level[p]
  DBuf<u32> gm;     // refined_community_mapping_per_level[p]
  DBuf<u32> s_pre;  // previous_subcommunity_mapping_per_level[p]
  DBuf<u32> s_cur;  // current_subcommunity_mapping_per_level[p]
  DBuf<double> k;   // weighted degree of each level-p node
  double tw = 0.0;  // 2m of G^p
};

// An edge list on the device (GraphInput): w == nullptr means weight 1.0.
struct DevEdges {
  const u32* u = nullptr;
  const u32* v = nullptr;
  const double* w = nullptr;
  u64 k = 0;
};

// Scratch reused by every stage; grown on demand, never shrunk.
struct Scratch {
  DBuf<u8> cub_tmp;
  // edge-list staging (host batches, aggregation output)
  DBuf<u32> eu, ev, eu2, ev2;
  DBuf<double> ew, ew2;
  // delta application
  DBuf<u64> keys, keys2, rkeys, rkeys2;
  DBuf<u32> idx, idx2, segid, seg_start, rvals, rvals2;
  DBuf<u8> op, touched, ktouched, isdel, isins;
  DBuf<double> neww;
  DBuf<u32> nops_del, nops_ins, pos_del, pos_ins;
  DBuf<u32> delpre, inspre;  // per-row operation ranges (start, end) of apply_delta
  DBuf<u32> opdel, opdelpre;  // apply_delta: delete flags of the sorted operations, their scan
  DBuf<int> ddeg;
  DBuf<u64> newoff;
  DBuf<u32> rowlist;
  // node flags (level size)
  DBuf<u8> active, next, changed, affected, refined;
  DBuf<u32> act, cand_idx, cnt;
  DBuf<u32> cand_to, cand_node;
  DBuf<double> cand_gain, cand_k;
  DBuf<u64> gkey, gkey2;
  DBuf<u32> sel_from, sel_to, sel_node, order, order2;
  DBuf<u8> status, nmask;
  DBuf<u32> role;
  DBuf<u64> res;
  DBuf<double> d;       // community degrees (2n)
  DBuf<u32> used, rank;
  // refinement
  DBuf<u32> par, uroot, csize, ncomp, newid, minmem;
  DBuf<u64> keep;
  DBuf<u8> affsc, cand_sc, blocked;
  DBuf<u32> sizes;
  DBuf<double> dS, wsp, dcomm;
  DBuf<u64> wcnt;       // T-filter: terms of each any-order sum
  DBuf<u8> amb;         // T-filter: S whose decision needs the ordered sum
  DBuf<u32> longrows;   // T-filter: member rows summed by a whole block
  DBuf<u32> upd_node, upd_to;
  // reductions
  DBuf<double> red, red2;
  DBuf<u64> red64;
  DBuf<u32> origin;
  // global tables of the block-per-vertex kernel's second pass (rows with
  // more than 2048 distinct keys)
  DBuf<u32> huge_key, huge_pos, huge_list;
  DBuf<u32> ovf, ovf_cnt;  // block kernel: rows deferred to the pass with global regions
  DBuf<u32> acc_cnt;       // inc-movement: accepted moves over all rounds
  DBuf<u32> hubk, hubk2, hubv;  // block bin ordered by degree (keys, sorted keys, list)
  DBuf<u32> foldseg, foldcnt;   // ordered sums: long segments, folded in runs, and their count
  DBuf<double> fvals;           // ordered sums: the terms gathered into sum order
  DBuf<double> huge_val;
  // deterministic mode (det.cu)
  DBuf<u32> det_bits, det_bp, det_keys, det_rsort, det_mkey, det_mkey2, det_mval, det_members,
      det_mstart, det_mcount, det_xhead, det_xnext;
  DBuf<double> det_bw, det_wsp;
  DBuf<u64> det_out, det_k64, det_k64b;
  DBuf<u8> det_wvalid;
  // partitioned second pass of the block kernel (integral weights)
  DBuf<u32> pb_nb, pb_nc, pb_bbase, pb_cbase, pb_rowfail, pb_fail, pb_failcnt, pb_ktmp, pb_ekey,
      pb_epos, pb_bcnt, pb_boff, pb_bp, pb_bk;
  DBuf<u64> pb_ne, pb_ebase, pb_ro0;
  DBuf<double> pb_wcur, pb_ew, pb_bg, pb_rkv, pb_rdcur;
  DBuf<u32> pb_brow, pb_crow, pb_rv, pb_rfv, pb_rcur;  // bucket / chunk -> row; row scalars
  DBuf<u32> pb_okey, pb_okey2, pb_oval, pb_ord, pb_fwork;  // fold order (largest bucket first)
  DBuf<unsigned long long> mark_long;  // (rank << 32 | segment) of long moved rows
  DBuf<u32> mark_long_cnt;
  // batch statistics accumulated on the device and read once at the end of
  // the call: [0..7] traversed / candidates of the four evaluation bins,
  // [8] accepted moves, [9] refinement merges, [10] |B^1|
  DBuf<u64> bacc;
  DBuf<u8> kflag;     // K marks for the next level (M8), level-size bytes
  DBuf<u32> kflag_ids;  // moved hubs whose rows k_mark_next_long marks
  // movement rounds of a small frontier (small.cu)
  DBuf<u32> sm_list_a, sm_list_b;
  DBuf<u64> sm_out;
  // per-level output: the level's s_cur before the batch, the changed nodes
  DBuf<u32> lvl_prev, lvl_nodes, lvl_ids;
  DBuf<u8> lvl_flag;
};

// Per-kernel device timing (CUDA events on the engine's stream), enabled by
// HL_FLAG_KERNEL_TIMING; bytes are the algorithmic bytes the stage moved.
struct KernelAgg {
  u64 launches = 0;
  double ms = 0.0;
  u64 bytes = 0;
  u64 items = 0;  // vertices / records processed, where meaningful
};
enum KernelId : int {
  KT_MOVE_EVAL = 0,
  KT_REFINE_EVAL,
  KT_SELECT,
  KT_MERGE_ROWS,
  KT_AGGREGATE,
  KT_EVAL_SMALL,   // sub-warp bins (both evaluation kinds)
  KT_EVAL_MID,     // warp-per-vertex bin
  KT_EVAL_BIG,     // warp-per-vertex wide bin (129..512)
  KT_EVAL_HUGE,    // block-per-vertex bin (> 512), both passes
  KT_COMM_DEG,     // per-community / per-sub-community degree sums
  KT_MARK_NEXT,    // accepted-move application and frontier marking
  KT_REFINE_CC,    // connected components of affected sub-communities
  KT_TFILTER,      // T-filter sums and decisions
  KT_ROW_SUMS,     // vertex degrees of touched rows
  KT_DELTA_SORT,   // batch key sort and resolution in apply_delta
  KT_STAGE_APPLY,  // whole stages of the level loop (including host waits)
  KT_STAGE_MOVE,
  KT_STAGE_REFINE,
  KT_STAGE_AGGREGATE,
  KT_HOST_SYNC,    // host waits on the stream (launches = count; no time)
  KT_COPY_ROWS,    // untouched CSR rows copied into the new buffer
  KT_MOVE_SMALL,   // movement rounds of a small frontier in one block (small.cu)
  KT_EVAL_PB,      // the partitioned pass of the block bin (inside KT_EVAL_HUGE)
  KT_COUNT
};

struct Engine {
  hl_config cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;
  MemCtx mem;
  Scratch sc;
  std::vector<Level> levels;
  bool multilevel = false;
  bool integral = true;  // every weight integral: all FP64 sums exact in any order
  bool in_bootstrap = false;  // hl_create's bootstrap is running
  HostScalars hs;
  u64 epoch = 1;         // selection epochs (reservation keys)
  u32 sel_round = 0;     // role tag of the current selection
  u64 stats_sel_iters = 0;
  u64 nlaunch = 0;       // launches of this library's kernels
  u64 launch_mark = 0;
  // per-call statistics
  hl_batch_stats st{};
  std::vector<std::pair<u32, u32>> new_ids;  // (new sub-community id, origin) of the last refinement
  // K marks handed to the next level's inc_movement (M8): the nodes it gained
  // from splits below and the nodes whose community the projection changed
  bool k_flags_set = false;
  u64 sum_nv_batch = 0;  // frontier sizes of the multi-kernel evaluations, this call
  // degree-bin thresholds picked by the autotuner (0 = compile-time default)
  struct Tune {
    u32 mid_max = 0, wide_max = 0;
    u32 hub_defer = 0;  // integral weights: hub rows above this many entries skip pass 1
    bool done = false;
    u32 frontier = 0;
    float best_ms = 0.f;
  } tune;
  // per-level output (hl_set_level_callback): called after each level's refinement
  hl_level_fn level_fn = nullptr;
  void* level_user = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // kernel timing
  bool ktiming = false;
  KernelAgg kagg[KT_COUNT];
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending;
  cudaEvent_t kt_begin();
  void kt_end(int id, cudaEvent_t a);
  void kt_collect();

  u64 read_u64(const u64* dptr);
  u32 read_u32(const u32* dptr);
  // Several device scalars with one wait: out[i] = *ptrs[i] (at most 16).
  void read_u32s(std::initializer_list<const u32*> ptrs, u32* out);
  double read_f64(const double* dptr);
  void sync();
};

// CUB helper: query temp bytes, grow the shared temp buffer, run.
template <typename F>
inline void cub_run(Engine& E, F f) {
  size_t bytes = 0;
  HL_CUDA(f((void*)nullptr, bytes));
  E.sc.cub_tmp.ensure(E.mem, bytes + 16);
  HL_CUDA(f((void*)E.sc.cub_tmp.p, bytes));
}

// ---- stage entry points (one .cu file each) --------------------------------
// graph.cu
void graph_init_empty(Engine& E, Level& L, u32 n);
void graph_grow_nodes(Engine& E, Level& L, u32 n);
void apply_delta(Engine& E, Level& L, const DevEdges& b, u32 new_n, bool keep_loops);
void recompute_all_degrees(Engine& E, Level& L);
double tree_sum(Engine& E, const double* x, u64 n);
void seq_sums(Engine& E, u32 nseg, const u64* off, const double* x, double init, int path,
              double* out);
// List (and zeroed count) for the long segments of one ordered-sum kernel
// pair: room for every segment of RUN_FOLD_MIN or more of `total` terms.
struct FoldList {
  u32* seg;
  u32* cnt;
};
FoldList fold_list(Engine& E, u64 total, u32 nseg);
bool edges_integral(Engine& E, const DevEdges& b);
void check_endpoints(Engine& E, const DevEdges& b, u32 n);

// move.cu
struct MoveOut {
  u32 iterations = 0;
  u64 moves = 0, candidates = 0, traversed = 0, changed = 0;
};
MoveOut inc_movement(Engine& E, Level& L, const DevEdges& delta, bool all_active,
                     bool mark_moved);
void recompute_comm_degrees(Engine& E, Level& L, const u32* part, u32 ncomm_cap, double* d);
void compact_labels_if_needed(Engine& E, u32* labels, u32 n, u32 limit);
void select_decoupled_dev(Engine& E, u32 M);
void ensure_comm_arrays(Engine& E, size_t ncap);
void run_eval(Engine& E, int kind, const u32* verts, u32 nv, const Level& L, const u32* s,
              const double* d, const u8* blocked, bool allow_empty, u32* out_to, double* out_gain,
              unsigned long long* traversed);

// refine.cu
struct RefineOut {
  u64 splits = 0, merges = 0, refined = 0;
  u64 tfilter_exact = 0;  // candidates decided from the ordered sum
  u32 smax_before = 0;
};
RefineOut inc_refinement(Engine& E, Level& L, bool cc_same_community);

// api.cu: device-side batch statistics (Scratch::bacc)
void stats_acc_u64(Engine& E, const unsigned long long* src, u32 count, u32 slot);
void stats_acc_u32(Engine& E, const u32* src, u32 slot);
void stats_count_flags(Engine& E, const u8* flags, u32 n, u32 slot);

// small.cu: movement rounds of a small frontier in one block.  Returns true
// when the movement stage is finished, false when the host rounds continue
// from S.active (*big_degree: an active vertex exceeds the block's tables).
bool move_rounds_small(Engine& E, Level& L, bool mark_moved, u32& it, u64& moves, u64& cands,
                       u64& trav, u64& sum_nv, bool* big_degree);

// eval.cu: degree-bin autotuner (once per handle)
void autotune_bins(Engine& E, const u32* verts, u32 nv, const Level& L, const u32* s,
                   const double* d, u32* out_to, double* out_gain);

// det.cu: the sequential (RunMode::Deterministic) steps
void inc_movement_det(Engine& E, Level& L, double* d, size_t dcap, bool mark_moved, u64* moves,
                      u64* traversed);
u64 merge_singletons_det(Engine& E, Level& L, const u32* rv, u32 nr, u32* sizes, double* dS,
                         const double* dcomm, size_t scap);

// Test switch: decide every T-filter candidate from the ordered sum.
extern std::atomic<int> g_exact_tfilter;
// Test switch: table slots of the partitioned hub pass (eval.cu).
extern std::atomic<u32> g_pb_slots;
extern std::atomic<u32> g_dbg_hub_defer;
extern std::atomic<u64> g_dbg_pb_round;

// aggregate.cu
u64 inc_aggregation(Engine& E, Level& L, const DevEdges& delta, u32* next_n,
                    bool changed_only, bool edge_weight_loops);  // output in sc.eu2/ev2/ew2
u64 aggregate_full(Engine& E, Level& L, const u32* s, u32* out_u, u32* out_v, double* out_w);
void project_up(Engine& E, Level& lo, Level& hi, u8* changed_flags = nullptr);
void top_down(Engine& E);
void inherit_new_nodes(Engine& E, Level& hi, const std::vector<std::pair<u32, u32>>& ids);

// modularity.cu
double modularity(Engine& E, Level& L, const u32* part);
void canonicalize_device(Engine& E, u32* labels, u64 n, u32* out);
u32 rank_compact(Engine& E, u32* labels, u32 n, u32 id_bound);

// kernels used by more than one stage
__global__ void k_fill_u8(u8* p, u8 v, u64 n);
__global__ void k_iota(u32* p, u32 n);

}  // namespace hl
