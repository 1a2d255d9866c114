"""RunMode::Deterministic on the GPU against the oracle's restatement of the
reference's sequential loops (hit_leiden.rs:1103-1191 movement, :1392-1548
singleton merges with the live T-filter).

The bar the path is held to is modularity within 2e-3 of the reference over
ten seeds; the GPU's sequential kernels follow the reference's step order, so
the maps come out bit-identical as well, and the tests check both.
"""
import importlib

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
gh = pytest.importorskip("tests.gpu_helpers")

hl = importlib.import_module("hit-leiden_b200")
W = importlib.import_module("hit-leiden_b200.workloads")
E2E = importlib.import_module("tests.test_gpu_e2e")

DET = hl.RunMode.Deterministic


def oracle_det(n, s, d, w, levels):
    if levels == 1:
        st = O.State(n, levels=1, mode=O.MODE_DETERMINISTIC)
        st.push_empty_graph()
        st.hit_leiden(s, d, w)
    else:
        st = O.State(n, mode=O.MODE_DETERMINISTIC)
        st.bootstrap(s, d, w, max_levels=levels)
    return st


@pytest.mark.parametrize("weights", [None, (0.5, 2.0)])
@pytest.mark.parametrize("levels", [1, 10])
@pytest.mark.parametrize("seed", range(10))
def test_deterministic_e2e_ten_seeds(seed, levels, weights):
    n, s, d, w, _ = W.planted(1500, 6.0, 0.2, seed, comm_min=5, comm_max=60, triangle_frac=0.2,
                              weights=weights)
    gs = hl.PartitionState.load(hl.GraphInput.from_arrays("det", n, s, d, w),
                                hl.RunConfig(max_iterations=levels))
    assert gs.config.mode == DET
    os_ = oracle_det(n, s, d, w, levels)
    E2E.compare(gs, os_)
    store = W.EdgeStore(n, s, d, w)
    for b in range(3):
        u, v, ww = W.mixed_batch(store, 150, 0.8, 300 + 10 * seed + b, weights=weights,
                                 preferential=True)
        it = hl.hit_leiden(gs, hl.GraphInput.from_arrays("d", n, u, v, ww), 1.0, DET)
        assert it == gs.levels  # one iteration per level, as the reference returns
        os_.hit_leiden(u, v, ww)
        E2E.compare(gs, os_)
        assert abs(gs.modularity() - os_.modularity(0)) <= 2e-3


def test_deterministic_rmat_hubs():
    n, bs, bd = W.rmat_torch(12, 16, 4, device="cpu")
    s = bs.numpy().view(np.uint32).copy()
    d = bd.numpy().view(np.uint32).copy()
    gs = hl.PartitionState.load(hl.GraphInput.from_arrays("rmat", n, s, d, None),
                                hl.RunConfig(max_iterations=10))
    os_ = oracle_det(n, s, d, np.ones(len(s)), 10)
    E2E.compare(gs, os_)
    for b in range(2):
        u, v, ww = W.rmat_batch_torch(12, bs, bd, 2000, 0.9, 60 + b)
        u, v, ww = u.numpy().view(np.uint32), v.numpy().view(np.uint32), ww.numpy()
        gs.apply_batch(u, v, ww)
        os_.hit_leiden(u, v, ww)
        E2E.compare(gs, os_)


def test_mode_switch_per_call():
    """hit_leiden takes the mode per call (hit_leiden.rs:940): a throughput
    bootstrap followed by a deterministic batch equals the oracle fed the
    same state and batch in deterministic mode."""
    n, s, d, w, _ = W.planted(1200, 6.0, 0.25, 11, comm_min=5, comm_max=60, triangle_frac=0.2)
    gs = hl.PartitionState.load(hl.GraphInput.from_arrays("t", n, s, d, w),
                                hl.RunConfig(mode=hl.RunMode.Throughput, max_iterations=10))
    levels = []
    for p in range(gs.levels):
        off, col, ww = gs.supergraph(p)
        levels.append({"off": off, "col": col, "w": ww,
                       "f": gs.community_mapping_per_level[p],
                       "g": gs.refined_community_mapping_per_level[p],
                       "s_pre": gs.previous_subcommunity_mapping_per_level[p],
                       "s_cur": gs.current_subcommunity_mapping_per_level[p]})
    os_ = O.State(n, levels=1, mode=O.MODE_DETERMINISTIC)
    os_.import_levels(levels)
    u, v, ww = W.uniform_inserts(n, 200, 5, set(zip(s.tolist(), d.tolist())))
    hl.hit_leiden(gs, hl.GraphInput.from_arrays("d", n, u, v, ww), 1.0, DET)
    os_.hit_leiden(u, v, ww)
    E2E.compare(gs, os_)


def _graph(n, edges):
    src = np.array([e[0] for e in edges], np.uint32)
    dst = np.array([e[1] for e in edges], np.uint32)
    w = np.array([e[2] for e in edges], np.float64)
    return O.Graph.from_edges(n, src, dst, w)


def test_deterministic_movement_considers_empty_community():
    # hit_leiden.rs:2016-2052 in deterministic mode: node 2 leaves for the
    # empty community at gamma = 3
    g = _graph(3, [(0, 1, 10.0), (0, 2, 0.5)])
    with gh.stage_mode(DET):
        f, _, _, it = gh.inc_movement(g, [], [], [], [0, 0, 0], [0, 0, 0], 3.0)
    assert f[2] != f[0] and it == 1
    fo, _, _, _ = O.inc_movement(g, [], [], None, [0, 0, 0], [0, 0, 0], 3.0,
                                 O.MODE_DETERMINISTIC)
    assert np.array_equal(f, fo)


def test_deterministic_refinement_t_filter():
    # hit_leiden.rs:2058-2114 in deterministic mode: the T-filter keeps node 2
    # out of sub-community {1}
    g = _graph(4, [(0, 1, 10.0), (0, 3, 100.0), (1, 3, 100.0), (1, 2, 1.0)])
    with gh.stage_mode(DET):
        s, _ = gh.inc_refinement(g, [0, 0, 0, 1], [0, 1, 2, 3], [True] * 4, 1.0)
    assert s[2] == 2
    so, _ = O.inc_refinement(g, [0, 0, 0, 1], [0, 1, 2, 3], [True] * 4, 1.0,
                             O.MODE_DETERMINISTIC)
    assert np.array_equal(s, so)


@pytest.mark.parametrize("weights", [None, (0.5, 2.0)])
@pytest.mark.parametrize("seed", range(4))
def test_deterministic_stages_bit_exact(seed, weights):
    """The two sequential stages alone on random snapshots, against the
    oracle's deterministic branches: movement from a perturbed partition with
    a delta, then refinement with the live T-filter."""
    n, s, d, w, _ = W.planted(2500, 8.0, 0.3, 50 + seed, comm_min=5, comm_max=80,
                              triangle_frac=0.2, weights=weights)
    g = O.Graph.from_edges(n, s, d, w)
    rng = np.random.default_rng(seed)
    f0 = O.run(n, s, d, w)[0].astype(np.uint32)
    f0[rng.choice(n, n // 10, replace=False)] = rng.integers(0, n, n // 10)
    s0 = np.arange(n, dtype=np.uint32)
    u, v, ww = W.uniform_inserts(n, 300, 9 + seed, set(zip(s.tolist(), d.tolist())))
    with gh.stage_mode(DET):
        f1, ch, af, _ = gh.inc_movement(g, u, v, ww, f0, s0, 1.0, mark_moved=True)
    fo, cho, afo, _ = O.inc_movement(g, u, v, ww, f0, s0, 1.0, O.MODE_DETERMINISTIC,
                                     mark_moved=True)
    assert np.array_equal(f1, fo) and np.array_equal(ch, cho) and np.array_equal(af, afo)
    # refinement from a coarse sub-community map inside the new communities
    sub = (f1.astype(np.int64) * 2 + (np.arange(n) % 2)).astype(np.uint32)
    for exact in (False, True):
        with gh.stage_mode(DET), gh.exact_tfilter(exact):
            s1, r1 = gh.inc_refinement(g, f1, sub, af, 1.0, cc_same_community=True)
        so, ro = O.inc_refinement(g, f1, sub, af, 1.0, O.MODE_DETERMINISTIC,
                                  cc_same_community=True)
        assert np.array_equal(s1, so) and np.array_equal(r1, ro)
