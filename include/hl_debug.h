/* hl_debug.h — function-level entry points of libhl used by the parity tests.
 *
 * Each call runs ONE stage of the update path on the GPU, on host-provided
 * inputs, with the same kernels the product path uses, so that every stage can
 * be compared with its reference counterpart on a fixed snapshot.  Graphs are
 * passed as canonical CSR (rows sorted by neighbour id, a self-loop twice in
 * its row).  All pointers are host pointers; outputs are caller-allocated.
 */
#ifndef HL_DEBUG_H
#define HL_DEBUG_H
#include "hl.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Per-vertex best move on a fixed snapshot (f, d(C), k, 2m):
 * parallel_frontier.rs:133-239 (`execute_shard`, one node).  out_to is the
 * chosen community (n+v for the empty community), out_gain its gain; a gain
 * <= 0 means no move. */
HL_API hl_status hl_dbg_move_eval(int32_t device, uint32_t n, const uint64_t* off, const uint32_t* col,
                           const double* w, const uint32_t* f, const double* d, uint64_t d_len,
                           const double* k, double tw, double gamma, const uint32_t* verts,
                           uint64_t nv, uint32_t* out_to, double* out_gain);

/* Decoupled move selection: throughput.rs:204-236 (`select_decoupled_moves`).
 * Writes the accepted nodes in selection order; *out_count their number. */
HL_API hl_status hl_dbg_select_decoupled(int32_t device, const uint32_t* node, const uint32_t* from,
                                  const uint32_t* to, const double* gain, uint64_t m,
                                  uint32_t* out_nodes, uint64_t* out_count);

/* G ⊕ ΔG: in_memory.rs:103-137 (`apply_delta`).  Returns the new CSR through
 * out_off (n_out+1 entries), out_col / out_w (capacity cap); *out_nnz entries. */
HL_API hl_status hl_dbg_apply_delta(int32_t device, uint32_t n, const uint64_t* off, const uint32_t* col,
                             const double* w, uint32_t delta_n, const uint32_t* dsrc,
                             const uint32_t* ddst, const double* dw, uint64_t dk,
                             int32_t keep_self_loops, uint64_t* out_off, uint32_t* out_col,
                             double* out_w, uint64_t cap, uint64_t* out_nnz);

/* inc_movement in the mode hl_dbg_set_mode selects (throughput by default):
 * hit_leiden.rs:1024-1101, deterministic :1103-1191.  f is updated in
 * place; changed / affected (may be NULL) receive B and K as 0/1 bytes. */
HL_API hl_status hl_dbg_inc_movement(int32_t device, uint32_t n, const uint64_t* off, const uint32_t* col,
                              const double* w, const uint32_t* dsrc, const uint32_t* ddst,
                              const double* dw, uint64_t dk, uint32_t* f, const uint32_t* s,
                              double gamma, uint32_t max_rounds, int32_t mark_moved,
                              uint8_t* changed, uint8_t* affected, uint32_t* iterations);

/* inc_refinement in the mode hl_dbg_set_mode selects (throughput by default,
 * deterministic merges hit_leiden.rs:1392-1548): hit_leiden.rs:1265-1390 with
 * throughput.rs:239-359.  s is updated in place; refined receives R. */
HL_API hl_status hl_dbg_inc_refinement(int32_t device, uint32_t n, const uint64_t* off,
                                const uint32_t* col, const double* w, const uint32_t* f,
                                uint32_t* s, const uint8_t* affected, double gamma,
                                int32_t cc_same_community, uint8_t* refined);

/* inc_aggregation: hit_leiden.rs:1639-1731.  Writes the compressed ΔH (ascending
 * (u,v), capacity cap), the updated s_pre and the next level's node count. */
HL_API hl_status hl_dbg_inc_aggregation(int32_t device, uint32_t n, const uint64_t* off,
                                 const uint32_t* col, const double* w, const uint32_t* dsrc,
                                 const uint32_t* ddst, const double* dw, uint64_t dk,
                                 const uint32_t* s_pre, const uint32_t* s_cur,
                                 const uint8_t* refined, int32_t changed_only,
                                 int32_t edge_weight_loops, uint32_t* out_s_pre,
                                 uint32_t* out_next_n, uint32_t* out_u, uint32_t* out_v,
                                 double* out_w, uint64_t cap, uint64_t* out_count);

/* The fixed-shape pairwise sum used for 2m (tiles of 1024, stride halving). */
HL_API hl_status hl_dbg_tree_sum(int32_t device, const double* x, uint64_t n, double* out);

/* Left-to-right f64 sums, out[i] = init + x[off[i]] + ... + x[off[i+1]-1]
 * with every addition rounded in that order: the fold behind the row sums
 * (hit_leiden.rs:1063), the community degrees and the aggregation's
 * per-super-edge sums.  path 0 is the library's own choice (runs of same-binade
 * terms for segments of 512 or more, one addition after another below), 1
 * always folds in runs, 2 never does; all three give the same bits.  No
 * reference counterpart: the entry point exposes the fold to tests. */
HL_API hl_status hl_dbg_seq_sums(int32_t device, uint32_t nseg, const uint64_t* off,
                                 const double* x, double init, int32_t path, double* out);

/* Test switch, process-wide: nonzero makes the refinement's T-filter decide
 * every candidate from the ordered sum w(S, C) (hit_leiden.rs:1618-1625)
 * instead of the any-order sum with its rounding window.  Results are the same
 * either way; the switch lets tests cover the ordered path.  No reference
 * counterpart. */
HL_API hl_status hl_dbg_set_exact_tfilter(int32_t on);

/* RunMode of the stage entry points above (hl_dbg_inc_movement,
 * hl_dbg_inc_refinement, ...): HL_MODE_THROUGHPUT (the default) or
 * HL_MODE_DETERMINISTIC, so that the reference's dual-mode tests
 * (dual_mode_test!, hit_leiden.rs:1823-1841) run on both GPU paths. */
HL_API hl_status hl_dbg_set_mode(uint32_t mode);

/* Table slots (64..512, 0 = 512) of the partitioned pass that evaluates
 * long hub rows under integral weights (rows above 8192 entries, or with
 * more than 2048 distinct neighbour keys).  A small table makes buckets
 * overflow, so tests reach the global-table pass those rows fall back to.
 * Results do not depend on it. */
HL_API hl_status hl_dbg_set_bucket_slots(uint32_t slots);

/* Integral weights: hub rows (above the wide bin) longer than `entries` go
 * straight to the partitioned pass instead of the block kernel's shared
 * tables (0 = each handle's bound: 8192, or the autotuner's pick).  Every
 * bound gives the same results; tests use it to send all hub rows through
 * either path. */
HL_API hl_status hl_dbg_set_hub_defer(uint32_t entries);

/* Entries the partitioned pass takes per round of its kernels (0 = 96 Mi).
 * Smaller rounds keep a round's keys and bucketed entries in L2 between the
 * scatter and the fold, at the price of more launches.  Results do not
 * depend on it. */
HL_API hl_status hl_dbg_set_pb_round(uint64_t entries);

/* Warp-bin thresholds of the stage entry points (mid_max in [33, 128],
 * wide_max in [mid_max, 512]; 0 = default), the pairs the autotuner picks
 * from.  Results do not depend on them. */
HL_API hl_status hl_dbg_set_bins(uint32_t mid_max, uint32_t wide_max);

/* Modularity of `part` on the CSR (hit_leiden.rs:121-161). */
HL_API hl_status hl_dbg_modularity(int32_t device, uint32_t n, const uint64_t* off, const uint32_t* col,
                            const double* w, const uint32_t* part, double* q);

#ifdef __cplusplus
}
#endif
#endif /* HL_DEBUG_H */
