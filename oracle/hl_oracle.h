/* hl_oracle.h — C interface of the CPU oracle (test infrastructure only).
 *
 * Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * through ctypes.  The product library (libhl) never links or calls it.
 */
#ifndef HL_ORACLE_H
#define HL_ORACLE_H
#include <stdint.h>

enum { OR_MODE_DETERMINISTIC = 0, OR_MODE_THROUGHPUT = 1 };

enum {
  OR_MAP_F = 0,      /* community_mapping_per_level            */
  OR_MAP_G = 1,      /* refined_community_mapping_per_level    */
  OR_MAP_S_PRE = 2,  /* previous_subcommunity_mapping_per_level */
  OR_MAP_S_CUR = 3,  /* current_subcommunity_mapping_per_level  */
  OR_MAP_NODE_TO_COMM = 4
};

enum {
  OR_FLAG_KEEP_SELF_LOOPS = 1u << 0,   /* apply_delta keeps existing self-loops   */
  OR_FLAG_AGG_CHANGED_ONLY = 1u << 1,  /* inc_aggregation iterates R ∩ changed    */
  OR_FLAG_EDGE_WEIGHT_LOOPS = 1u << 2, /* self-loop transfer moves w, not 2w      */
  OR_FLAG_NO_COMPACT = 1u << 3,        /* never compact community ids >= n        */
  OR_FLAG_FAITHFUL_SCANS = 1u << 4,    /* T-filter with the reference's O(n) scans */
  OR_FLAG_MULTILEVEL = 1u << 5,        /* multi-level update semantics (M1-M7)    */
  OR_FLAG_HUB_CHECK = 1u << 6          /* check round-to-round hub key sums (below) */
};

/* Throughput movement with OR_FLAG_HUB_CHECK also evaluates every active row
 * of more than 512 entries a second way: from a table of (key, sum, first
 * position) per row, built at the row's first evaluation in the movement
 * call and corrected after each round by the moves of its neighbours (first
 * positions recomputed only when a key that lost its first entry ties the
 * best gain).  Each such evaluation is compared with the full one.  This
 * returns and resets the counters: evaluations, mismatches, first-position
 * rescans, corrections, table builds, keys scanned.  Test infrastructure:
 * the results of the update do not depend on the flag. */
void or_hub_check_counters(uint64_t out[6]);
/* The check's stale first-position path on a fixed case: the number of
 * rescans it made (1 expected), or -1 if an evaluation differed. */
int or_hub_check_selftest(void);

typedef struct or_graph or_graph;
typedef struct or_state or_state;

typedef struct {
  uint32_t iterations;
  uint64_t moves, candidates, traversed, splits, merges, changed, refined;
} or_stats;

or_graph* or_graph_from_edges(uint32_t n, const uint32_t* src, const uint32_t* dst, const double* w,
                              uint64_t m);
void or_graph_free(or_graph* g);
uint32_t or_graph_nodes(const or_graph* g);
uint64_t or_graph_entries(const or_graph* g);
void or_graph_csr(const or_graph* g, uint64_t* off, uint32_t* col, double* w);
or_graph* or_graph_apply_delta(const or_graph* g, uint32_t delta_n, const uint32_t* src,
                               const uint32_t* dst, const double* w, uint64_t k, int keep_loops);
void or_node_degrees(const or_graph* g, double* out);
double or_twice_total_weight(const or_graph* g);
double or_tree_sum(const double* x, uint64_t n);
double or_modularity_edges(uint32_t n, const uint32_t* src, const uint32_t* dst, const double* w,
                           uint64_t m, const uint32_t* part);
double or_modularity_csr(const or_graph* g, const uint32_t* part);
void or_canonicalize(uint32_t* c, uint64_t n);
uint64_t or_select_decoupled(const uint32_t* node, const uint32_t* from, const uint32_t* to,
                             const double* kdeg, const double* gain, uint64_t m,
                             uint32_t* out_nodes);
void or_move_eval(const or_graph* g, const uint32_t* f, const double* d, uint64_t d_len,
                  const double* k, double tw, double gamma, const uint32_t* verts, uint64_t nv,
                  uint32_t* out_to, double* out_gain);
uint32_t or_inc_movement(const or_graph* g, const uint32_t* dsrc, const uint32_t* ddst,
                         const double* dw, uint64_t dk, uint32_t* f, const uint32_t* s,
                         double gamma, int mode, uint32_t max_rounds, int compact, int mark_moved,
                         uint8_t* out_changed, uint8_t* out_affected);
void or_inc_refinement(const or_graph* g, const uint32_t* f, uint32_t* s, const uint8_t* affected,
                       double gamma, int mode, int faithful, int cc_same_community,
                       uint8_t* out_refined);
uint64_t or_inc_aggregation(const or_graph* g, const uint32_t* dsrc, const uint32_t* ddst,
                            const double* dw, uint64_t dk, const uint32_t* s_pre,
                            const uint32_t* s_cur, const uint8_t* refined, uint32_t flags,
                            uint32_t* out_s_pre, uint32_t* out_next_n, uint32_t* out_u,
                            uint32_t* out_v, double* out_w, uint64_t cap);
void or_def_update(uint32_t P, const uint32_t* sizes, uint32_t* f_cat, const uint32_t* s_cat,
                   uint8_t* changed_cat);

or_state* or_state_new(uint32_t n, uint32_t levels, double gamma, int mode, uint32_t flags,
                       uint32_t max_rounds);
void or_state_free(or_state* s);
void or_state_push_empty_graph(or_state* s, uint32_t n);
int or_hit_leiden(or_state* s, uint32_t delta_n, const uint32_t* src, const uint32_t* dst,
                  const double* w, uint64_t k, or_stats* stats);
uint32_t or_state_levels(const or_state* s);
void or_state_import_begin(or_state* s, uint32_t levels, uint32_t flags);
int or_state_import_level(or_state* s, uint32_t level, uint32_t n, const uint64_t* off,
                          const uint32_t* col, const double* w, const uint32_t* f,
                          const uint32_t* g, const uint32_t* s_pre, const uint32_t* s_cur);
int or_state_bootstrap(or_state* s, uint32_t n, const uint32_t* src, const uint32_t* dst,
                       const double* w, uint64_t m, uint32_t max_levels, or_stats* stats);
uint32_t or_state_level_nodes(const or_state* s, uint32_t level, int which);
int or_state_get_map(const or_state* s, uint32_t level, int which, uint32_t* out);
int or_state_set_map(or_state* s, uint32_t level, int which, const uint32_t* in, uint32_t n);
const or_graph* or_state_graph(or_state* s, uint32_t level);
double or_state_modularity(const or_state* s, uint32_t level, int which);
double or_run(uint32_t n, const uint32_t* src, const uint32_t* dst, const double* w, uint64_t m,
              double gamma, uint32_t max_levels, uint64_t seed, uint32_t* out_part,
              uint32_t* out_levels);

/* Host threads the throughput-mode snapshot evaluations use (default: the
 * hardware concurrency, at most 64; 0 restores the default). */
int or_num_threads(void);
void or_set_num_threads(int threads);

#endif
