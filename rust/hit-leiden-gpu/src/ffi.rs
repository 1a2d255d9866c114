//! Raw declarations of the C ABI in `include/hl.h`, field for field and entry
//! point for entry point.  Every function returns an `hl_status` (`i32`);
//! `hl_last_error()` holds the calling thread's last message.
#![allow(non_camel_case_types)]

use std::os::raw::{c_char, c_void};

pub type hl_status = i32;
pub const HL_OK: hl_status = 0;
pub const HL_ERR_INVALID_INPUT: hl_status = 1;
pub const HL_ERR_CUDA: hl_status = 2;
pub const HL_ERR_OUT_OF_MEMORY: hl_status = 3;
pub const HL_ERR_TIMEOUT: hl_status = 4;
pub const HL_ERR_UNSUPPORTED: hl_status = 5;

pub const HL_MODE_DETERMINISTIC: u32 = 0;
pub const HL_MODE_THROUGHPUT: u32 = 1;

pub const HL_MAP_COMMUNITY: u32 = 0;
pub const HL_MAP_REFINED: u32 = 1;
pub const HL_MAP_SUB_PREVIOUS: u32 = 2;
pub const HL_MAP_SUB_CURRENT: u32 = 3;

pub const HL_FLAG_KEEP_SELF_LOOPS: u32 = 1 << 0;
pub const HL_FLAG_BATCH_MODULARITY: u32 = 1 << 1;
pub const HL_FLAG_KERNEL_TIMING: u32 = 1 << 2;
pub const HL_FLAG_NO_AUTOTUNE: u32 = 1 << 3;
pub const HL_FLAG_NO_SMALL_ROUNDS: u32 = 1 << 4;

pub const HL_NOALLOC_MAX_ELEMS: u64 = 1 << 28;

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct hl_config {
    pub resolution: f64,
    pub mode: u32,
    pub max_levels: u32,
    pub max_rounds: u32,
    pub flags: u32,
    pub hbm_budget: u64,
    pub device: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct hl_batch_stats {
    pub iterations: u32,
    pub levels: u32,
    pub moves: u64,
    pub candidates: u64,
    pub traversed: u64,
    pub splits: u64,
    pub merges: u64,
    pub changed: u64,
    pub refined: u64,
    pub edges: u64,
    pub modularity: f64,
    pub device_ms: f64,
    pub launches: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct hl_kernel_stat {
    pub name: [c_char; 32],
    pub launches: u64,
    pub total_ms: f64,
    pub bytes: u64,
    pub items: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct hl_request_done {
    pub request_id: u64,
    pub batch_id: u64,
    pub batch_seq: u64,
    pub edges: u64,
    pub batch_edges: u64,
    pub changed: u64,
    pub modularity: f64,
    pub queue_ms: f64,
    pub service_ms: f64,
    pub latency_ms: f64,
    pub graph: u32,
    pub batch_requests: u32,
    pub status: i32,
    pub pad_: u32,
    pub level0_ms: f64,
}

/// Per-level output callback (`hl_level_fn`).
pub type hl_level_fn = Option<unsafe extern "C" fn(user: *mut c_void, level: u32, count: u64,
                                                    nodes: *const u32, sub_ids: *const u32)>;
/// Per-level output callback of the server (`hl_server_level_fn`).
pub type hl_server_level_fn = Option<unsafe extern "C" fn(user: *mut c_void, graph: u32,
                                                           batch_id: u64, level: u32, count: u64,
                                                           nodes: *const u32,
                                                           sub_ids: *const u32)>;

/// Opaque graph handle.
#[repr(C)]
pub struct hl_graph {
    _private: [u8; 0],
}

/// Opaque server handle.
#[repr(C)]
pub struct hl_server {
    _private: [u8; 0],
}

extern "C" {
    pub fn hl_config_default(cfg: *mut hl_config) -> hl_status;
    pub fn hl_create(cfg: *const hl_config, n: u32, src: *const u32, dst: *const u32,
                     w: *const f64, m: u64, out: *mut *mut hl_graph) -> hl_status;
    pub fn hl_create_device(cfg: *const hl_config, n: u32, d_src: *const u32,
                            d_dst: *const u32, d_w: *const f64, m: u64,
                            out: *mut *mut hl_graph) -> hl_status;
    pub fn hl_apply_batch(g: *mut hl_graph, src: *const u32, dst: *const u32, w: *const f64,
                          k: u64, stats: *mut hl_batch_stats) -> hl_status;
    pub fn hl_apply_batch_device(g: *mut hl_graph, d_src: *const u32, d_dst: *const u32,
                                 d_w: *const f64, k: u64, stats: *mut hl_batch_stats)
                                 -> hl_status;
    pub fn hl_kernel_stats(g: *const hl_graph, out: *mut hl_kernel_stat, cap: u32,
                           count: *mut u32) -> hl_status;
    pub fn hl_reset_kernel_stats(g: *mut hl_graph) -> hl_status;
    pub fn hl_set_resolution(g: *mut hl_graph, gamma: f64) -> hl_status;
    pub fn hl_set_mode(g: *mut hl_graph, mode: u32) -> hl_status;
    pub fn hl_autotune_info(g: *const hl_graph, mid_max: *mut u32, wide_max: *mut u32,
                            hub_defer: *mut u32, frontier: *mut u32) -> hl_status;
    pub fn hl_set_level_callback(g: *mut hl_graph, fn_: hl_level_fn, user: *mut c_void)
                                 -> hl_status;
    pub fn hl_num_nodes(g: *const hl_graph, n: *mut u32) -> hl_status;
    pub fn hl_num_levels(g: *const hl_graph, levels: *mut u32) -> hl_status;
    pub fn hl_level_size(g: *const hl_graph, level: u32, n_level: *mut u32) -> hl_status;
    pub fn hl_num_edges(g: *const hl_graph, level: u32, entries: *mut u64) -> hl_status;
    pub fn hl_get_partition(g: *const hl_graph, out: *mut u32) -> hl_status;
    pub fn hl_get_map(g: *const hl_graph, level: u32, which: u32, out: *mut u32) -> hl_status;
    pub fn hl_get_csr(g: *const hl_graph, level: u32, off: *mut u64, col: *mut u32,
                      w: *mut f64) -> hl_status;
    pub fn hl_modularity(g: *const hl_graph, q: *mut f64) -> hl_status;
    pub fn hl_modularity_of(g: *const hl_graph, part: *const u32, q: *mut f64) -> hl_status;
    pub fn hl_canonicalize(device: i32, labels: *mut u32, n: u64) -> hl_status;
    pub fn hl_destroy(g: *mut hl_graph);
    pub fn hl_device_bytes(g: *const hl_graph, used: *mut u64, peak: *mut u64) -> hl_status;

    pub fn hl_apply_batches(graphs: *const *mut hl_graph, src: *const *const u32,
                            dst: *const *const u32, w: *const *const f64, k: *const u64,
                            count: u32, workers: u32, statuses: *mut hl_status,
                            stats: *mut hl_batch_stats) -> hl_status;

    pub fn hl_server_create(workers: u32, hbm_budget: u64, out: *mut *mut hl_server)
                            -> hl_status;
    pub fn hl_server_add_graph(s: *mut hl_server, g: *mut hl_graph, graph_id: *mut u32)
                               -> hl_status;
    pub fn hl_server_set_edge_estimate(s: *mut hl_server, bytes_per_edge: u64) -> hl_status;
    pub fn hl_server_set_coalescing(s: *mut hl_server, max_requests: u32) -> hl_status;
    pub fn hl_server_submit(s: *mut hl_server, graph_id: u32, src: *const u32, dst: *const u32,
                            w: *const f64, k: u64, request_id: *mut u64) -> hl_status;
    pub fn hl_server_poll(s: *mut hl_server, out: *mut hl_request_done, cap: u32,
                          count: *mut u32, wait_ms: i32) -> hl_status;
    pub fn hl_server_set_level_callback(s: *mut hl_server, fn_: hl_server_level_fn,
                                        user: *mut c_void) -> hl_status;
    pub fn hl_server_drain(s: *mut hl_server) -> hl_status;
    pub fn hl_server_destroy(s: *mut hl_server);

    pub fn hl_last_error() -> *const c_char;
    pub fn hl_version() -> *const c_char;

    pub fn hl_tree_sum_noalloc(d_x: *const f64, n: u64, d_out: *mut f64, stream: *mut c_void)
                               -> hl_status;
}
