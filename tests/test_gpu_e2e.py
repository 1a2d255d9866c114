"""End-to-end parity: a GPU-resident state driven through the C ABI (hl_create +
hl_apply_batch) against the oracle state fed the same graph and batches.

Bit-exact: every per-level map (f, g, s_pre, s_cur) and every level's CSR after
the bootstrap and after each batch.  Modularity within 1e-12 relative.
"""
import importlib

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
gh = pytest.importorskip("tests.gpu_helpers")

hl = importlib.import_module("hit-leiden_b200")
W = importlib.import_module("hit-leiden_b200.workloads")


def oracle_state(n, src, dst, w, levels):
    if levels == 1:
        st = O.State(n, levels=1, mode=O.MODE_THROUGHPUT)
        st.push_empty_graph()
        st.hit_leiden(src, dst, w)
    else:
        st = O.State(n, mode=O.MODE_THROUGHPUT)
        st.bootstrap(src, dst, w, max_levels=levels)
    return st


def compare(gs, os_, check_csr=True):
    P = os_.levels
    assert gs.levels == P
    maps = [(O.MAP_F, gs.community_mapping_per_level), (O.MAP_G,
            gs.refined_community_mapping_per_level),
            (O.MAP_S_PRE, gs.previous_subcommunity_mapping_per_level),
            (O.MAP_S_CUR, gs.current_subcommunity_mapping_per_level)]
    for which, got in maps:
        for p in range(P):
            exp = os_.get_map(p, which)
            assert np.array_equal(got[p], exp), f"map {which} level {p} differs"
    if check_csr:
        for p in range(P):
            off, col, w = gs.supergraph(p)
            ro, rc, rw = os_.graph(p).csr()
            assert np.array_equal(off, ro) and np.array_equal(col, rc)
            assert np.array_equal(w.view(np.uint64), rw.view(np.uint64)), f"weights level {p}"
    q_o = os_.modularity(0)
    q_g = gs.modularity()
    assert abs(q_o - q_g) <= 1e-12 * max(1.0, abs(q_o))


def small_planted(seed, n=2000, weights=None):
    n, s, d, w, _ = W.planted(n, 6.0, 0.2, seed, comm_min=5, comm_max=80, triangle_frac=0.2,
                              weights=weights)
    return n, s, d, w


@pytest.mark.parametrize("levels", [1, 10])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_e2e_unit_weights_inserts(levels, seed):
    n, s, d, w = small_planted(seed)
    cfg = hl.RunConfig(mode=hl.RunMode.Throughput, max_iterations=levels)
    gs = hl.PartitionState.load(hl.GraphInput.from_arrays("t", n, s, d, w), cfg)
    os_ = oracle_state(n, s, d, w, levels)
    compare(gs, os_)
    ex = set(zip(s.tolist(), d.tolist()))
    for b in range(4):
        u, v, ww = W.uniform_inserts(n, 200, 1000 * seed + b, ex)
        gs.apply_batch(u, v, ww)
        os_.hit_leiden(u, v, ww)
        compare(gs, os_)


@pytest.mark.parametrize("levels", [1, 10])
@pytest.mark.parametrize("seed", [0, 1])
@pytest.mark.parametrize("exact", [False, True])
def test_e2e_f64_weights_mixed(levels, seed, exact):
    with gh.exact_tfilter(exact):
        _f64_weights_mixed(levels, seed)


def _f64_weights_mixed(levels, seed):
    n, s, d, w = small_planted(seed, weights=(0.5, 2.0))
    cfg = hl.RunConfig(mode=hl.RunMode.Throughput, max_iterations=levels)
    gs = hl.PartitionState.load(hl.GraphInput.from_arrays("t", n, s, d, w), cfg)
    os_ = oracle_state(n, s, d, w, levels)
    compare(gs, os_)
    store = W.EdgeStore(n, s, d, w)
    for b in range(4):
        u, v, ww = W.mixed_batch(store, 300, 0.9, 77 + b, weights=(0.5, 2.0))
        gs.apply_batch(u, v, ww)
        os_.hit_leiden(u, v, ww)
        compare(gs, os_)


def test_e2e_config1_shape():
    n, s, d, w = W.config1(0)
    gs = hl.PartitionState.load(hl.GraphInput.from_arrays("c1", n, s, d, w), hl.RunConfig(mode=hl.RunMode.Throughput))
    os_ = oracle_state(n, s, d, w, 10)
    compare(gs, os_)
    ex = set(zip(s.tolist(), d.tolist()))
    for b in range(5):
        u, v, ww = W.uniform_inserts(n, 1000, 100 + b, ex)
        gs.apply_batch(u, v, ww)
        os_.hit_leiden(u, v, ww)
        compare(gs, os_)


def test_e2e_deletes_and_empty_batch():
    n, s, d, w = small_planted(5)
    gs = hl.PartitionState.load(hl.GraphInput.from_arrays("t", n, s, d, w), hl.RunConfig(mode=hl.RunMode.Throughput))
    os_ = oracle_state(n, s, d, w, 10)
    # delete 100 existing edges exactly, then an empty batch (all vertices active)
    idx = np.random.default_rng(0).choice(len(s), 100, replace=False)
    gs.apply_batch(s[idx], d[idx], -w[idx])
    os_.hit_leiden(s[idx], d[idx], -w[idx])
    compare(gs, os_)
    gs.apply_batch([], [], [])
    os_.hit_leiden([], [], [])
    compare(gs, os_)


def test_reference_hit_leiden_api_mirror():
    # hit_leiden.rs:3136-3177: strong cross edges must not increase the count.
    e = [(0, 1, 10.0), (1, 2, 10.0), (0, 2, 10.0), (3, 4, 10.0), (4, 5, 10.0), (3, 5, 10.0),
         (2, 3, 0.1)]
    st = hl.PartitionState.load(hl.GraphInput("t", 6, e), hl.RunConfig(mode=hl.RunMode.Throughput, max_iterations=1))
    c0 = len(set(st.community_mapping_per_level[0].tolist()))
    it = hl.hit_leiden(st, hl.GraphInput("d", 6, [(0, 3, 100.0), (1, 4, 100.0)]), 1.0,
                       hl.RunMode.Throughput)
    assert it >= 1
    assert np.array_equal(st.node_to_comm, st.refined_community_mapping_per_level[0])
    assert len(set(st.community_mapping_per_level[0].tolist())) <= max(c0, 6)
    off, col, w = st.supergraph(0)
    nb0 = dict(zip(col[off[0]:off[1]].tolist(), w[off[0]:off[1]].tolist()))
    assert nb0[3] == 100.0


def test_errors_are_reported_not_raised_across_abi():
    with pytest.raises(hl.HitLeidenError) as e:
        hl.PartitionState.load(hl.GraphInput("t", 3, [(0, 5, None)]))
    assert e.value.kind == "InvalidInput"
    # the reference's default mode runs on the GPU too
    det = hl.PartitionState.load(hl.GraphInput("t", 3, [(0, 1, None)]))
    assert det.config.mode == hl.RunMode.Deterministic and det.levels >= 1
    det.close()
    with pytest.raises(hl.HitLeidenError) as e:
        hl.RunConfig(max_iterations=0).validate()
    assert e.value.kind == "InvalidInput"
    st = hl.PartitionState.load(hl.GraphInput("t", 3, [(0, 1, None)]))
    with pytest.raises(hl.HitLeidenError) as e:
        st.apply_batch([0], [9], [1.0])
    assert e.value.kind == "InvalidInput"
    # the handle stays usable after a rejected batch
    st.apply_batch([1], [2], [1.0])
    assert st.supergraph(0)[0][-1] == 4


def test_hbm_budget_is_enforced():
    n, s, d, w = small_planted(0)
    with pytest.raises(hl.HitLeidenError) as e:
        hl.PartitionState.load(hl.GraphInput.from_arrays("t", n, s, d, w),
                               hl.RunConfig(mode=hl.RunMode.Throughput, hbm_budget=64 * 1024))
    assert e.value.kind == "OutOfMemory"


def test_empty_and_tiny_graphs():
    for n, edges in [(1, []), (4, []), (2, [(0, 1, None)]), (3, [(0, 0, 2.0), (1, 2, None)])]:
        for lv in [1, 10]:
            g = hl.GraphInput("t", n, edges)
            st = hl.PartitionState.load(g, hl.RunConfig(mode=hl.RunMode.Throughput, max_iterations=lv))
            src, dst, w = g.arrays()
            os_ = oracle_state(n, src, dst, w, lv)
            compare(st, os_)


@pytest.mark.parametrize("seed", [0, 1])
def test_e2e_rmat_integral_hubs(seed):
    """Skewed R-MAT degrees with unit weights (the large plain configuration's
    shape, scale 12): GPU state bit-exact with the oracle after the bootstrap
    and after mixed batches of R-MAT inserts and deletes."""
    import torch
    n, bs, bd = W.rmat_torch(12, 16, seed, device="cuda:0")
    s = bs.cpu().numpy().view(np.uint32)
    d = bd.cpu().numpy().view(np.uint32)
    w = np.ones(len(s))
    gs = hl.PartitionState.load(hl.GraphInput.from_arrays("rmat", n, s, d, None),
                                hl.RunConfig(mode=hl.RunMode.Throughput, max_iterations=10))
    os_ = oracle_state(n, s, d, w, 10)
    compare(gs, os_)
    for b in range(3):
        u, v, ww = W.rmat_batch_torch(12, bs, bd, 2000, 0.9, 100 * seed + b)
        u = u.cpu().numpy().view(np.uint32)
        v = v.cpu().numpy().view(np.uint32)
        ww = ww.cpu().numpy()
        gs.apply_batch(u, v, ww)
        os_.hit_leiden(u, v, ww)
        compare(gs, os_)
    del torch


@pytest.mark.parametrize("weights", [None, (0.5, 2.0)])
def test_small_frontier_rounds_change_nothing(weights):
    """Rounds of a small frontier run whole in one block (small.cu); with that
    path off every round takes the multi-kernel path.  Both give the same
    state, bit for bit, and both equal the oracle."""
    n, s, d, w, _ = W.planted(6000, 8.0, 0.25, 13, comm_min=5, comm_max=80, triangle_frac=0.2,
                              weights=weights)
    on = hl.PartitionState.load(hl.GraphInput.from_arrays("t", n, s, d, w),
                                hl.RunConfig(mode=hl.RunMode.Throughput))
    off = hl.PartitionState.load(hl.GraphInput.from_arrays("t", n, s, d, w),
                                 hl.RunConfig(mode=hl.RunMode.Throughput, small_rounds=False))
    os_ = oracle_state(n, s, d, w, 10)
    store = W.EdgeStore(n, s, d, w)
    for b in range(4):
        u, v, ww = W.mixed_batch(store, 300, 0.8, 40 + b, weights=weights, preferential=True)
        st_on = on.apply_batch(u, v, ww)
        st_off = off.apply_batch(u, v, ww)
        os_.hit_leiden(u, v, ww)
        assert st_on.iterations == st_off.iterations and st_on.moves == st_off.moves
        compare(on, os_)
        compare(off, os_)
    on.close()
    off.close()
