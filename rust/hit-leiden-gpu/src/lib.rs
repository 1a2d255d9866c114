//! GPU drop-in for the incremental update path of the `hit_leiden` crate.
//!
//! The reference crate updates a `PartitionState` in place with
//! `hit_leiden(&mut state, &delta, gamma, mode) -> usize`
//! (src/core/algorithm/hit_leiden.rs:936-941) and exposes the hierarchy through
//! the state's `pub` vectors (src/core/partition/state.rs:19-32).  Here the
//! state lives on one B200 behind the `libhl` handle: [`PartitionState::load`]
//! loads a graph and builds the hierarchy, [`hit_leiden`] applies one
//! edge-update batch, and the accessors read the per-level maps back.
//!
//! Types keep the reference's names and meaning: [`GraphInput`]
//! (src/core/types.rs:133-147; a `None` weight is 1.0, a negative weight
//! weakens or deletes), [`RunMode`] (src/core/config.rs:19-23), [`RunConfig`]
//! (config.rs:25-51, with `max_iterations` as the level cap) and
//! [`HitLeidenError`] (src/core/error.rs:19-27).  Nothing panics across the
//! boundary: every failure comes back as an error value.
pub mod ffi;

use std::ffi::CStr;
use std::fmt;
use std::ptr;

/// Edge list or edge delta (src/core/types.rs:133-147).
#[derive(Clone, Debug, PartialEq)]
pub struct GraphInput {
    pub dataset_id: String,
    pub node_count: usize,
    pub edges: Vec<(usize, usize, Option<f64>)>,
}

impl GraphInput {
    pub fn empty(dataset_id: impl Into<String>) -> Self {
        GraphInput { dataset_id: dataset_id.into(), node_count: 0, edges: Vec::new() }
    }
}

/// src/core/config.rs:19-23.
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum RunMode {
    Deterministic,
    Throughput,
}

/// The part of `RunConfig` (config.rs:25-51) the update path reads, plus the
/// device-side settings of the handle.
#[derive(Clone, Debug, PartialEq)]
pub struct RunConfig {
    pub mode: RunMode,
    pub quality_tolerance: f64,
    /// Level cap of the hierarchy (1 = the reference's single-level state).
    pub max_iterations: usize,
    pub resolution: f64,
    /// Throughput movement round cap (hit_leiden.rs:1077).
    pub max_rounds: u32,
    /// Device bytes the handle may hold; 0 = no cap.
    pub hbm_budget: u64,
    pub device: i32,
}

impl Default for RunConfig {
    /// The reference's defaults (config.rs:37-48): deterministic mode, 10
    /// iterations, resolution 1.0, tolerance 0.001.
    fn default() -> Self {
        RunConfig {
            mode: RunMode::Deterministic,
            quality_tolerance: 0.001,
            max_iterations: 10,
            resolution: 1.0,
            max_rounds: 20,
            hbm_budget: 0,
            device: 0,
        }
    }
}

impl RunConfig {
    /// config.rs:54-61.
    pub fn validate(&self) -> Result<(), String> {
        if self.max_iterations == 0 {
            return Err("max_iterations must be > 0".to_string());
        }
        if self.quality_tolerance < 0.0 {
            return Err("quality_tolerance must be >= 0".to_string());
        }
        Ok(())
    }
}

/// src/core/error.rs:19-27, with the library's status codes mapped onto it.
#[derive(Debug, Clone, PartialEq)]
pub enum HitLeidenError {
    InvalidInput(String),
    Backend(String),
    Acceleration(String),
}

impl fmt::Display for HitLeidenError {
    fn fmt(&self, f: &mut fmt::Formatter<'_>) -> fmt::Result {
        match self {
            HitLeidenError::InvalidInput(m) => write!(f, "invalid input: {}", m),
            HitLeidenError::Backend(m) => write!(f, "backend error: {}", m),
            HitLeidenError::Acceleration(m) => write!(f, "acceleration error: {}", m),
        }
    }
}

impl std::error::Error for HitLeidenError {}

fn last_error() -> String {
    unsafe {
        let p = ffi::hl_last_error();
        if p.is_null() {
            String::new()
        } else {
            CStr::from_ptr(p).to_string_lossy().into_owned()
        }
    }
}

fn check(rc: ffi::hl_status) -> Result<(), HitLeidenError> {
    match rc {
        ffi::HL_OK => Ok(()),
        ffi::HL_ERR_INVALID_INPUT => Err(HitLeidenError::InvalidInput(last_error())),
        ffi::HL_ERR_CUDA | ffi::HL_ERR_OUT_OF_MEMORY | ffi::HL_ERR_TIMEOUT => {
            Err(HitLeidenError::Acceleration(format!("status {}: {}", rc, last_error())))
        }
        _ => Err(HitLeidenError::Backend(format!("status {}: {}", rc, last_error()))),
    }
}

fn mode_code(mode: RunMode) -> u32 {
    match mode {
        RunMode::Deterministic => ffi::HL_MODE_DETERMINISTIC,
        RunMode::Throughput => ffi::HL_MODE_THROUGHPUT,
    }
}

/// Structure-of-arrays form of an edge list, as the C ABI takes it.  Fails on
/// an endpoint that does not fit the 32-bit ids of the device layout.
fn split_edges(edges: &[(usize, usize, Option<f64>)])
               -> Result<(Vec<u32>, Vec<u32>, Vec<f64>), HitLeidenError> {
    let mut src = Vec::with_capacity(edges.len());
    let mut dst = Vec::with_capacity(edges.len());
    let mut w = Vec::with_capacity(edges.len());
    for &(u, v, x) in edges {
        if u > u32::MAX as usize || v > u32::MAX as usize {
            return Err(HitLeidenError::InvalidInput(format!(
                "endpoint ({}, {}) exceeds the 32-bit vertex ids of the device layout", u, v)));
        }
        src.push(u as u32);
        dst.push(v as u32);
        w.push(x.unwrap_or(1.0)); // None => 1.0 (in_memory.rs:49)
    }
    Ok((src, dst, w))
}

/// Statistics of one update batch (`hl_batch_stats`).
pub type BatchStats = ffi::hl_batch_stats;

/// A hierarchical partition resident on one GPU: the device counterpart of
/// the reference's `PartitionState` (state.rs:19-32).
pub struct PartitionState {
    g: *mut ffi::hl_graph,
    node_count: usize,
}

// The handle may move between threads; it is used by one thread at a time.
unsafe impl Send for PartitionState {}

impl PartitionState {
    /// Loads `graph` onto `config.device` and builds the bootstrap hierarchy
    /// (up to `config.max_iterations` levels).  Endpoints >= node_count are
    /// rejected, as `run()` rejects them (hit_leiden.rs:35-43).
    pub fn load(graph: &GraphInput, config: &RunConfig) -> Result<Self, HitLeidenError> {
        config.validate().map_err(HitLeidenError::InvalidInput)?;
        if graph.node_count > u32::MAX as usize {
            return Err(HitLeidenError::InvalidInput("node_count exceeds 32-bit ids".into()));
        }
        let (src, dst, w) = split_edges(&graph.edges)?;
        let mut c = ffi::hl_config::default();
        check(unsafe { ffi::hl_config_default(&mut c) })?;
        c.resolution = config.resolution;
        c.mode = mode_code(config.mode);
        c.max_levels = config.max_iterations.min(u32::MAX as usize) as u32;
        c.max_rounds = config.max_rounds;
        c.hbm_budget = config.hbm_budget;
        c.device = config.device;
        let mut g = ptr::null_mut();
        check(unsafe {
            ffi::hl_create(&c, graph.node_count as u32, src.as_ptr(), dst.as_ptr(), w.as_ptr(),
                           src.len() as u64, &mut g)
        })?;
        Ok(PartitionState { g, node_count: graph.node_count })
    }

    /// Applies one edge-update batch; returns the statistics of the batch.
    pub fn apply_batch(&mut self, delta: &GraphInput, gamma: f64, mode: RunMode)
                       -> Result<BatchStats, HitLeidenError> {
        let (src, dst, w) = split_edges(&delta.edges)?;
        check(unsafe { ffi::hl_set_resolution(self.g, gamma) })?;
        check(unsafe { ffi::hl_set_mode(self.g, mode_code(mode)) })?;
        let mut st = BatchStats::default();
        check(unsafe {
            ffi::hl_apply_batch(self.g, src.as_ptr(), dst.as_ptr(), w.as_ptr(),
                                src.len() as u64, &mut st)
        })?;
        Ok(st)
    }

    pub fn node_count(&self) -> usize {
        self.node_count
    }

    /// Number of levels in the hierarchy (`state.levels`).
    pub fn levels(&self) -> Result<usize, HitLeidenError> {
        let mut p = 0u32;
        check(unsafe { ffi::hl_num_levels(self.g, &mut p) })?;
        Ok(p as usize)
    }

    fn map(&self, level: usize, which: u32) -> Result<Vec<usize>, HitLeidenError> {
        let mut n = 0u32;
        check(unsafe { ffi::hl_level_size(self.g, level as u32, &mut n) })?;
        let mut out = vec![0u32; n as usize];
        check(unsafe { ffi::hl_get_map(self.g, level as u32, which, out.as_mut_ptr()) })?;
        Ok(out.into_iter().map(|x| x as usize).collect())
    }

    /// `community_mapping_per_level[level]` (f).
    pub fn community_mapping(&self, level: usize) -> Result<Vec<usize>, HitLeidenError> {
        self.map(level, ffi::HL_MAP_COMMUNITY)
    }

    /// `refined_community_mapping_per_level[level]` (g).
    pub fn refined_community_mapping(&self, level: usize) -> Result<Vec<usize>, HitLeidenError> {
        self.map(level, ffi::HL_MAP_REFINED)
    }

    /// `previous_subcommunity_mapping_per_level[level]` (s_pre).
    pub fn previous_subcommunity_mapping(&self, level: usize)
                                         -> Result<Vec<usize>, HitLeidenError> {
        self.map(level, ffi::HL_MAP_SUB_PREVIOUS)
    }

    /// `current_subcommunity_mapping_per_level[level]` (s_cur).
    pub fn current_subcommunity_mapping(&self, level: usize)
                                        -> Result<Vec<usize>, HitLeidenError> {
        self.map(level, ffi::HL_MAP_SUB_CURRENT)
    }

    /// Node-indexed community partition, relabelled 0..k-1 in first-seen
    /// order (`canonicalized_community_ids`, hit_leiden.rs:358-376).
    pub fn partition(&self) -> Result<Vec<usize>, HitLeidenError> {
        let mut out = vec![0u32; self.node_count];
        check(unsafe { ffi::hl_get_partition(self.g, out.as_mut_ptr()) })?;
        Ok(out.into_iter().map(|x| x as usize).collect())
    }

    /// CSR of level `level` (`state.supergraphs[level]`): offsets, neighbours
    /// and weights, rows sorted by neighbour id.
    pub fn supergraph(&self, level: usize)
                      -> Result<(Vec<u64>, Vec<u32>, Vec<f64>), HitLeidenError> {
        let mut n = 0u32;
        let mut m = 0u64;
        check(unsafe { ffi::hl_level_size(self.g, level as u32, &mut n) })?;
        check(unsafe { ffi::hl_num_edges(self.g, level as u32, &mut m) })?;
        let mut off = vec![0u64; n as usize + 1];
        let mut col = vec![0u32; m as usize];
        let mut w = vec![0f64; m as usize];
        check(unsafe {
            ffi::hl_get_csr(self.g, level as u32, off.as_mut_ptr(), col.as_mut_ptr(),
                            w.as_mut_ptr())
        })?;
        Ok((off, col, w))
    }

    /// Modularity of the level-0 community partition (compute_modularity,
    /// hit_leiden.rs:121-161).
    pub fn modularity(&self) -> Result<f64, HitLeidenError> {
        let mut q = 0.0;
        check(unsafe { ffi::hl_modularity(self.g, &mut q) })?;
        Ok(q)
    }

    /// Device bytes held now and at most since creation.
    pub fn device_bytes(&self) -> Result<(u64, u64), HitLeidenError> {
        let (mut used, mut peak) = (0u64, 0u64);
        check(unsafe { ffi::hl_device_bytes(self.g, &mut used, &mut peak) })?;
        Ok((used, peak))
    }
}

impl Drop for PartitionState {
    fn drop(&mut self) {
        unsafe { ffi::hl_destroy(self.g) }
    }
}

/// `hit_leiden(&mut state, &delta, gamma, mode) -> usize`
/// (hit_leiden.rs:936-941): applies `delta` and returns the movement rounds
/// summed over the levels.
pub fn hit_leiden(state: &mut PartitionState, delta: &GraphInput, gamma: f64, mode: RunMode)
                  -> Result<usize, HitLeidenError> {
    Ok(state.apply_batch(delta, gamma, mode)?.iterations as usize)
}

/// Version string of the loaded library.
pub fn version() -> String {
    unsafe { CStr::from_ptr(ffi::hl_version()).to_string_lossy().into_owned() }
}

#[cfg(test)]
mod tests {
    use super::*;

    #[test]
    fn config_defaults_follow_the_reference() {
        let c = RunConfig::default();
        assert_eq!(c.mode, RunMode::Deterministic);
        assert_eq!(c.max_iterations, 10);
        assert_eq!(c.resolution, 1.0);
        assert!(c.validate().is_ok());
        assert!(RunConfig { max_iterations: 0, ..RunConfig::default() }.validate().is_err());
    }

    #[test]
    fn split_edges_defaults_missing_weights_to_one() {
        let (s, d, w) = split_edges(&[(0, 1, None), (1, 2, Some(-1.0))]).unwrap();
        assert_eq!(s, vec![0, 1]);
        assert_eq!(d, vec![1, 2]);
        assert_eq!(w, vec![1.0, -1.0]);
    }

    /// Needs a B200: HL_GPU_TESTS=1 cargo test.
    #[test]
    fn two_triangles_update_on_the_gpu() {
        if std::env::var("HL_GPU_TESTS").is_err() {
            return;
        }
        let g = GraphInput {
            dataset_id: "two-triangles".into(),
            node_count: 6,
            edges: vec![(0, 1, None), (1, 2, None), (0, 2, None), (3, 4, None), (4, 5, None),
                        (3, 5, None), (2, 3, None)],
        };
        let cfg = RunConfig { mode: RunMode::Throughput, ..RunConfig::default() };
        let mut st = PartitionState::load(&g, &cfg).unwrap();
        let q0 = st.modularity().unwrap();
        let delta = GraphInput { dataset_id: "d".into(), node_count: 6,
                                 edges: vec![(2, 3, Some(-1.0))] };
        hit_leiden(&mut st, &delta, 1.0, RunMode::Throughput).unwrap();
        let q1 = st.modularity().unwrap();
        assert!(q1 >= q0);
        assert_eq!(st.partition().unwrap().len(), 6);
    }
}
