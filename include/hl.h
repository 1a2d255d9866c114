/* hl.h — C ABI of the B200 HIT-Leiden incremental update path.
 *
 * A graph lives on one GPU behind an opaque handle.  The caller loads it once
 * (hl_create: load + bootstrap partition), then applies edge-update batches
 * (hl_apply_batch) and reads back the hierarchical partition and modularity.
 *
 * The reference crate (Rust `hit_leiden` 0.1.0) has no FFI; these entry points
 * replace its crate-level API for this path:
 *   hl_create        ~ PartitionState::identity + InMemoryGraph::from + the
 *                      first hit_leiden call (src/core/partition/state.rs:35-49,
 *                      src/core/graph/in_memory.rs:30-72,
 *                      src/core/algorithm/hit_leiden.rs:936-1018)
 *   hl_apply_batch   ~ hit_leiden(&mut state, &delta, gamma, mode)
 *                      (src/core/algorithm/hit_leiden.rs:936-941)
 *   hl_get_partition ~ reading PartitionState's per-level vectors
 *                      (src/core/partition/state.rs:19-32)
 *   hl_modularity    ~ compute_modularity (src/core/algorithm/hit_leiden.rs:121-161)
 *   hl_canonicalize  ~ canonicalize_community_ids_in_place (hit_leiden.rs:358-376)
 * Error codes mirror HitLeidenError::InvalidInput (src/core/error.rs:19-27) and
 * the endpoint check of run() (hit_leiden.rs:35-43); nothing panics or aborts
 * across this boundary.
 *
 * Conventions: host buffers are copied in; output buffers are caller-allocated.
 * A handle may be used by one thread at a time; different handles may be used
 * concurrently (each owns its own CUDA stream).
 */
#ifndef HL_H
#define HL_H
#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define HL_API __attribute__((visibility("default")))
#else
#define HL_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  HL_OK = 0,
  HL_ERR_INVALID_INPUT = 1, /* bad argument, endpoint >= n, bad config      */
  HL_ERR_CUDA = 2,          /* CUDA runtime / kernel launch failure          */
  HL_ERR_OUT_OF_MEMORY = 3, /* device allocation failed or HBM budget hit    */
  HL_ERR_TIMEOUT = 4,       /* a bounded device wait gave up                 */
  HL_ERR_UNSUPPORTED = 5    /* mode / feature not available on this path     */
} hl_status;

/* RunMode (src/core/config.rs:19-23).  Both run on the GPU.  Deterministic
 * (the reference's default) is the sequential Gauss–Seidel movement and the
 * sequential singleton merges (hit_leiden.rs:1103-1191, :1392-1548), run as
 * one persistent block per stage; Throughput is the round-based parallel form
 * (hit_leiden.rs:1068-1101, throughput.rs:80-359) and the fast path. */
typedef enum { HL_MODE_DETERMINISTIC = 0, HL_MODE_THROUGHPUT = 1 } hl_mode;

/* Which per-level map hl_get_map returns (state.rs:19-32). */
typedef enum {
  HL_MAP_COMMUNITY = 0,      /* f^p  community_mapping_per_level            */
  HL_MAP_REFINED = 1,        /* g^p  refined_community_mapping_per_level    */
  HL_MAP_SUB_PREVIOUS = 2,   /* s_pre^p previous_subcommunity_mapping       */
  HL_MAP_SUB_CURRENT = 3     /* s_cur^p current_subcommunity_mapping        */
} hl_map;

typedef struct {
  double resolution;    /* gamma (RunConfig.resolution, config.rs:35); default 1.0 */
  uint32_t mode;        /* hl_mode; default HL_MODE_DETERMINISTIC (config.rs:40-43) */
  uint32_t max_levels;  /* 1 = the reference's single-level state (state.rs:42);   */
                        /* >1 = multi-level bootstrap, levels created on demand    */
                        /* up to this cap (default 10, RunConfig.max_iterations)   */
  uint32_t max_rounds;  /* throughput movement round cap (hit_leiden.rs:1077); 20  */
  uint32_t flags;       /* HL_FLAG_*                                               */
  uint64_t hbm_budget;  /* bytes this handle may allocate on the device; 0 = no cap */
  int32_t device;       /* CUDA device ordinal                                     */
} hl_config;

/* Keep existing self-loops on apply_delta.  Off (the reference's behaviour,
 * in_memory.rs:122-130 keeps node < neighbor only) for max_levels == 1; the
 * multi-level mode always keeps them. */
#define HL_FLAG_KEEP_SELF_LOOPS (1u << 0)
/* Compute the level-0 modularity after every batch into hl_batch_stats
 * (an extra pass over the graph; off by default). */
#define HL_FLAG_BATCH_MODULARITY (1u << 1)
/* Time the main kernels with CUDA events on the handle's stream and count
 * their algorithmic bytes (read with hl_kernel_stats). */
#define HL_FLAG_KERNEL_TIMING (1u << 2)
/* Keep the compile-time degree bins instead of autotuning them.  By default
 * the first movement round after the bootstrap with at least 20,000 active
 * vertices runs the evaluation once per candidate pair of warp-bin
 * thresholds (results are identical for every pair) and keeps the fastest
 * pair for the handle (hl_autotune_info). */
#define HL_FLAG_NO_AUTOTUNE (1u << 3)
/* Keep every throughput movement round on the multi-kernel path.  By default
 * rounds whose frontier has at most 4096 vertices of at most 256 entries each
 * (levels of up to 2^18 nodes) run whole inside one block, without host round
 * trips between them; the results are identical either way. */
#define HL_FLAG_NO_SMALL_ROUNDS (1u << 4)

typedef struct {
  uint32_t iterations;   /* movement rounds summed over levels (hit_leiden return) */
  uint32_t levels;       /* levels in the state                                    */
  uint64_t moves;        /* accepted movement moves, all levels                    */
  uint64_t candidates;   /* positive-gain candidates, all levels                   */
  uint64_t traversed;    /* adjacency entries scanned by movement, all levels      */
  uint64_t splits;       /* sub-community components split off                     */
  uint64_t merges;       /* singleton refinement merges                            */
  uint64_t changed;      /* |B^1| level-0 vertices whose community changed         */
  uint64_t refined;      /* |R^1| level-0 vertices refined                         */
  uint64_t edges;        /* undirected edges in G^1 after the batch                */
  double modularity;     /* Q of the level-0 community partition after the batch   */
  double device_ms;      /* device time of the update, from the batch resident on  */
                         /* the device to the end (CUDA events; the host copy of   */
                         /* a host batch is excluded)                              */
  uint64_t launches;     /* kernels of this library launched by the call           */
} hl_batch_stats;

/* Accumulated per-kernel device time and algorithmic bytes. */
typedef struct {
  char name[32];
  uint64_t launches;
  double total_ms;
  uint64_t bytes;   /* algorithmic bytes, where counted            */
  uint64_t items;   /* vertices / records processed, where counted */
} hl_kernel_stat;

typedef struct hl_graph hl_graph;

/* Default configuration, RunConfig::default() (config.rs:37-48): gamma 1,
 * deterministic mode, 10 levels; 20 throughput rounds. */
HL_API hl_status hl_config_default(hl_config* cfg);

/* Load an undirected weighted graph of n vertices (m edges; w == NULL means
 * every weight is 1.0, as GraphInput's None weight, in_memory.rs:49) and build
 * the bootstrap partition.  Edges with an endpoint >= n are rejected. */
HL_API hl_status hl_create(const hl_config* cfg, uint32_t n, const uint32_t* src, const uint32_t* dst,
                    const double* w, uint64_t m, hl_graph** out);

/* Same, but src/dst/w are device pointers on cfg->device (no host copies). */
HL_API hl_status hl_create_device(const hl_config* cfg, uint32_t n, const uint32_t* d_src,
                           const uint32_t* d_dst, const double* d_w, uint64_t m,
                           hl_graph** out);

/* Apply one edge-update batch (GraphInput delta encoding, types.rs:133-147:
 * positive weight adds or strengthens, negative weakens or deletes; an edge
 * whose weight falls to <= 1e-12 is removed) and update the partition.
 * w == NULL means all weights are +1.0.  stats may be NULL.
 * A batch with an endpoint >= the node count is rejected with
 * HL_ERR_INVALID_INPUT before anything changes; the handle stays usable.
 * HL_ERR_OUT_OF_MEMORY or HL_ERR_CUDA from inside the update can leave some
 * levels updated and others not: the handle's state is then unspecified, and
 * the caller destroys it and loads the graph again. */
HL_API hl_status hl_apply_batch(hl_graph* g, const uint32_t* src, const uint32_t* dst, const double* w,
                         uint64_t k, hl_batch_stats* stats);

/* Same with device pointers (on the handle's device). */
HL_API hl_status hl_apply_batch_device(hl_graph* g, const uint32_t* d_src, const uint32_t* d_dst,
                                const double* d_w, uint64_t k, hl_batch_stats* stats);

/* Per-kernel statistics since creation or the last reset (needs
 * HL_FLAG_KERNEL_TIMING; otherwise launches stay 0).  *count receives the
 * number of entries; at most cap are written. */
HL_API hl_status hl_kernel_stats(const hl_graph* g, hl_kernel_stat* out, uint32_t cap,
                                 uint32_t* count);
HL_API hl_status hl_reset_kernel_stats(hl_graph* g);

/* Change gamma for subsequent batches (hit_leiden takes it per call,
 * hit_leiden.rs:939). */
HL_API hl_status hl_set_resolution(hl_graph* g, double gamma);

/* Per-level output: the reference's goal of emitting stabilised communities
 * as soon as they are ready instead of after the whole pass (README.md,
 * "Incremental community output"; no entry point in the crate).  While a
 * callback is set, hl_apply_batch calls it once per level, in level order,
 * right after that level's refinement: from there on the batch no longer
 * changes the level's sub-community map (s_cur^p, the refined communities
 * whose summaries a pipeline builds bottom-up).  It receives the level-p
 * nodes whose sub-community changed in this batch and their new
 * sub-community ids, in ascending node order (host arrays, valid during the
 * call only).  The communities f^p of every level are final when
 * hl_apply_batch returns.  Each call costs one device→host copy of the
 * level's changes.  fn == NULL turns it off.  The callback runs on the thread
 * that applies the batch and must not call back into this handle. */
typedef void (*hl_level_fn)(void* user, uint32_t level, uint64_t count, const uint32_t* nodes,
                            const uint32_t* sub_ids);
HL_API hl_status hl_set_level_callback(hl_graph* g, hl_level_fn fn, void* user);

/* Degree-bin thresholds the handle uses: vertices of degree 33..mid_max take
 * the warp kernel with a shared table, mid_max+1..wide_max the wide warp
 * kernel, larger ones the block kernel.  hub_defer (may be NULL): with
 * integral weights, hub rows longer than this go straight to the partitioned
 * pass (1: every row of the block bin).  frontier is the frontier size the autotuner measured on (0: not
 * tuned yet, or HL_FLAG_NO_AUTOTUNE). */
HL_API hl_status hl_autotune_info(const hl_graph* g, uint32_t* mid_max, uint32_t* wide_max,
                                  uint32_t* hub_defer, uint32_t* frontier);

/* Change the RunMode for subsequent batches (hit_leiden takes it per call,
 * hit_leiden.rs:940): HL_MODE_DETERMINISTIC or HL_MODE_THROUGHPUT. */
HL_API hl_status hl_set_mode(hl_graph* g, uint32_t mode);

HL_API hl_status hl_num_nodes(const hl_graph* g, uint32_t* n);
HL_API hl_status hl_num_levels(const hl_graph* g, uint32_t* levels);
HL_API hl_status hl_level_size(const hl_graph* g, uint32_t level, uint32_t* n_level);
HL_API hl_status hl_num_edges(const hl_graph* g, uint32_t level, uint64_t* entries);

/* Node-indexed community partition of the input vertices (f^1 after
 * def-update), relabelled to 0..k-1 in first-seen order; out has n entries. */
HL_API hl_status hl_get_partition(const hl_graph* g, uint32_t* out);

/* Raw per-level map (no relabelling); out has hl_level_size(level) entries. */
HL_API hl_status hl_get_map(const hl_graph* g, uint32_t level, uint32_t which, uint32_t* out);

/* CSR of level `level`: off has n_level+1 entries, col/w hl_num_edges entries.
 * Rows are sorted by neighbour id; a self-loop appears twice in its row. */
HL_API hl_status hl_get_csr(const hl_graph* g, uint32_t level, uint64_t* off, uint32_t* col,
                     double* w);

/* Modularity of the level-0 community partition (compute_modularity). */
HL_API hl_status hl_modularity(const hl_graph* g, double* q);

/* Modularity of an arbitrary node-indexed partition of the level-0 graph. */
HL_API hl_status hl_modularity_of(const hl_graph* g, const uint32_t* part, double* q);

/* First-seen contiguous relabelling of n labels, on the GPU of `device`. */
HL_API hl_status hl_canonicalize(int32_t device, uint32_t* labels, uint64_t n);

HL_API void hl_destroy(hl_graph* g);

/* Device bytes the handle holds now and at most since creation. */
HL_API hl_status hl_device_bytes(const hl_graph* g, uint64_t* used, uint64_t* peak);

/* ---- Many graphs on one GPU (no reference counterpart: the reference
 * updates one PartitionState per call) ------------------------------------
 *
 * Batching form.  Apply batch i (src[i], dst[i], w[i] — w may be NULL, or
 * w[i] NULL for all-ones — of k[i] edges, host arrays) to graphs[i], for all
 * i at once: up to `workers` host threads (0 = 16) each drive one graph at a
 * time on that graph's own stream, so the graphs' kernels and round trips
 * overlap on the GPU.  Each graph ends exactly as hl_apply_batch would leave
 * it.  A handle may appear once per call.  statuses (may be NULL) receives
 * each graph's status, stats (may be NULL) each graph's batch statistics;
 * the return value is the first failing status (HL_OK if none). */
HL_API hl_status hl_apply_batches(hl_graph* const* graphs, const uint32_t* const* src,
                                  const uint32_t* const* dst, const double* const* w,
                                  const uint64_t* k, uint32_t count, uint32_t workers,
                                  hl_status* statuses, hl_batch_stats* stats);

/* Serving form: a request loop over resident graphs.
 *   - A request (edges for one registered graph, host arrays, copied at
 *     submit) is admitted when the graphs' device bytes plus the estimates of
 *     admitted, unfinished requests (bytes_per_edge × edges, default 512)
 *     stay within hbm_budget (0 = no limit); a request that cannot fit even
 *     with nothing in flight completes with HL_ERR_OUT_OF_MEMORY.
 *   - `workers` threads update different graphs concurrently.  All requests
 *     admitted for a graph while it is busy are coalesced into its next batch,
 *     in arrival order; a graph's batches are applied one after another.
 *   - Each request completes with an hl_request_done record (hl_server_poll).
 *   - A failed batch leaves its graph as hl_apply_batch would, and the
 *     server keeps applying later requests to it.  After HL_ERR_OUT_OF_MEMORY
 *     or HL_ERR_CUDA in a record the caller drains the server, destroys it
 *     and reloads that graph.
 * The server does not own the graph handles: destroy it before them. */
typedef struct hl_server hl_server;
typedef struct {
  uint64_t request_id;
  uint64_t batch_id;       /* server-wide batch number                          */
  uint64_t batch_seq;      /* this graph's batch number, 1, 2, ... in order     */
  uint64_t edges;          /* edges of this request                             */
  uint64_t batch_edges;    /* edges of the coalesced batch it was applied in    */
  uint64_t changed;        /* |B^1| of that batch                               */
  double modularity;       /* NaN unless the graph has HL_FLAG_BATCH_MODULARITY */
  double queue_ms;         /* submit -> its batch started                       */
  double service_ms;       /* its batch started -> finished                     */
  double latency_ms;       /* submit -> finished                                */
  uint32_t graph;          /* graph id from hl_server_add_graph                 */
  uint32_t batch_requests; /* requests coalesced into that batch                */
  int32_t status;          /* hl_status of the batch                            */
  uint32_t pad_;
  double level0_ms;        /* submit -> its batch's level-0 sub-communities     */
                           /* settled (NaN without a server level callback)     */
} hl_request_done;

HL_API hl_status hl_server_create(uint32_t workers, uint64_t hbm_budget, hl_server** out);
HL_API hl_status hl_server_add_graph(hl_server* s, hl_graph* g, uint32_t* graph_id);
HL_API hl_status hl_server_set_edge_estimate(hl_server* s, uint64_t bytes_per_edge);
/* At most max_requests requests per coalesced batch (0 = all pending, the
 * default; 1 = every request is its own batch). */
HL_API hl_status hl_server_set_coalescing(hl_server* s, uint32_t max_requests);
HL_API hl_status hl_server_submit(hl_server* s, uint32_t graph_id, const uint32_t* src,
                                  const uint32_t* dst, const double* w, uint64_t k,
                                  uint64_t* request_id);
/* Up to cap completed requests (oldest first) into out; *count receives how
 * many.  wait_ms: 0 = do not wait, < 0 = wait until one completes or nothing
 * is outstanding, > 0 = wait at most that long. */
HL_API hl_status hl_server_poll(hl_server* s, hl_request_done* out, uint32_t cap, uint32_t* count,
                                int32_t wait_ms);
/* Per-level output of the served batches: fn gets the graph id and the
 * batch id with each level's changed sub-communities (hl_set_level_callback),
 * from the worker thread applying the batch, before the batch's requests
 * complete; level0_ms in the completion records then says when level 0 was
 * ready.  Set it before submitting; fn == NULL turns it off.  The server sets
 * the level callback of its graphs' handles while it holds them, and clears
 * it when it is destroyed. */
typedef void (*hl_server_level_fn)(void* user, uint32_t graph, uint64_t batch_id, uint32_t level,
                                   uint64_t count, const uint32_t* nodes, const uint32_t* sub_ids);
HL_API hl_status hl_server_set_level_callback(hl_server* s, hl_server_level_fn fn, void* user);
/* Wait until every submitted request has completed. */
HL_API hl_status hl_server_drain(hl_server* s);
/* Waits for outstanding requests, then stops the workers. */
HL_API void hl_server_destroy(hl_server* s);

/* Message for the last error on this thread (empty string if none). */
HL_API const char* hl_last_error(void);

/* Version string of the library build. */
HL_API const char* hl_version(void);

/* The canonical 2m reduction (fixed-shape pairwise sum: tiles of 1024 values
 * padded with +0.0, each folded by stride halving, the tile sums folded again)
 * of n doubles at device address d_x, written to the device address d_out, on
 * `stream` (a cudaStream_t; NULL = default stream) of the current device.
 * No counterpart in the reference: it exists for callers that must not
 * allocate device memory (an embedding runtime that owns all device memory, a
 * caller in a region where cudaMalloc is forbidden).  It allocates nothing:
 * its tile sums live in a fixed ~2 MB array compiled into the library, which
 * every GPU that loads the library keeps until exit.  n must not exceed
 * HL_NOALLOC_MAX_ELEMS (HL_ERR_INVALID_INPUT otherwise).  All calls on one GPU
 * share that array: calls whose work overlaps on the GPU race and must be
 * ordered by the caller.  Each call made outside stream capture resolves the
 * array's device address (cudaGetSymbolAddress) and keeps it for the device; a
 * call on a capturing stream uses the kept address, so make the first call on
 * a device before any stream capture.  The address lives as long as the
 * primary context: after cudaDeviceReset, make an uncaptured call again before
 * capturing one. */
#define HL_NOALLOC_MAX_ELEMS (1ull << 28)
HL_API hl_status hl_tree_sum_noalloc(const double* d_x, uint64_t n, double* d_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* HL_H */
