"""Pin the CPU oracle against the reference crate's own unit-test known answers.

Each test restates one assertion block of the reference's tests in
``src/core/algorithm/hit_leiden.rs`` (lines cited per test) or
``src/core/algorithm/throughput.rs``.  Tests marked with both modes mirror the
reference's ``dual_mode_test!`` macro (hit_leiden.rs:1823-1841).
"""
import numpy as np
import pytest

from oracle import oracle as O

MODES = [O.MODE_DETERMINISTIC, O.MODE_THROUGHPUT]


def unit(edges):
    src = [e[0] for e in edges]
    dst = [e[1] for e in edges]
    return src, dst, [1.0] * len(edges)


def weighted(edges):
    return [e[0] for e in edges], [e[1] for e in edges], [float(e[2]) for e in edges]


# --- apply_delta (hit_leiden.rs:1847-1897) ---------------------------------
def test_apply_delta_adds_edges():
    g = O.Graph.from_edges(4, *unit([(0, 1), (1, 2), (0, 2)]))
    up = g.apply_delta(*weighted([(2, 3, 1.0)]))
    assert 2 in [n for n, _ in up.neighbors(3)]
    assert 3 in [n for n, _ in up.neighbors(2)]
    assert abs(up.total_weight() - g.total_weight() - 1.0) < 1e-9


def test_apply_delta_removes_edges():
    g = O.Graph.from_edges(3, *unit([(0, 1), (1, 2), (0, 2)]))
    up = g.apply_delta(*weighted([(0, 2, -1.0)]))
    nb0 = [n for n, _ in up.neighbors(0)]
    assert 2 not in nb0 and 1 in nb0


def test_apply_delta_drops_existing_self_loops_and_keeps_delta_loops():
    # in_memory.rs:122-130 keeps node < neighbor only: an existing self-loop is
    # dropped by the next apply_delta, a self-loop in the delta survives.
    g = O.Graph.from_edges(3, *weighted([(0, 0, 5.0), (0, 1, 1.0)]))
    assert [n for n, _ in g.neighbors(0)] == [0, 0, 1]
    up = g.apply_delta(*weighted([(2, 2, 3.0)]))
    assert [n for n, _ in up.neighbors(0)] == [1]
    assert up.neighbors(2) == [(2, 3.0), (2, 3.0)]
    kept = g.apply_delta(*weighted([(2, 2, 3.0)]), keep_self_loops=True)
    assert [n for n, _ in kept.neighbors(0)] == [0, 0, 1]


def test_apply_delta_filters_small_weights_and_sums_in_order():
    g = O.Graph.from_edges(3, *weighted([(0, 1, 1.0), (1, 2, 2.0)]))
    up = g.apply_delta(*weighted([(1, 0, -1.0), (2, 1, 0.5), (1, 2, 0.25)]))
    assert up.neighbors(0) == []
    assert up.neighbors(1) == [(2, 2.75)]


# --- Algorithm 6 applies ΔG (hit_leiden.rs:1930-1971) ----------------------
@pytest.mark.parametrize("mode", MODES)
def test_hit_leiden_applies_delta_to_supergraph(mode):
    edges = [(0, 1), (1, 2), (0, 2), (3, 4), (4, 5), (3, 5), (2, 3)]
    st = O.State(6, mode=mode)
    # The reference test pushes From(initial) and then applies `initial` again.
    g0 = O.Graph.from_edges(6, *unit(edges))
    st.push_empty_graph()
    st.hit_leiden(*unit(edges))
    st.hit_leiden(*unit(edges))
    del g0
    st.hit_leiden(*weighted([(0, 5, 10.0)]))
    nb0 = dict(st.graph(0).neighbors(0))
    assert 5 in nb0 and abs(nb0[5] - 10.0) < 1e-9


# --- output = g¹ (hit_leiden.rs:1977-2010) ---------------------------------
@pytest.mark.parametrize("mode", MODES)
def test_hit_leiden_uses_refined_mapping(mode):
    edges = [(0, 1), (1, 2), (0, 2), (3, 4), (4, 5), (3, 5), (6, 7), (2, 3), (5, 6)]
    st = O.State(8, mode=mode)
    st.push_empty_graph()
    st.hit_leiden(*unit(edges))
    assert np.array_equal(st.get_map(0, O.MAP_NODE_TO_COMM), st.get_map(0, O.MAP_G))


# --- ∅ candidate at γ=3 (hit_leiden.rs:2016-2052) --------------------------
@pytest.mark.parametrize("mode", MODES)
def test_movement_considers_empty_community(mode):
    g = O.Graph.from_edges(3, *weighted([(0, 1, 10.0), (0, 2, 0.5)]))
    f, ch, k, it = O.inc_movement(g, [], [], [], [0, 0, 0], [0, 0, 0], 3.0, mode)
    assert f[2] != f[0]


# --- T-filter (hit_leiden.rs:2058-2114) -------------------------------------
@pytest.mark.parametrize("mode", MODES)
def test_refinement_t_filter_excludes_well_connected_subcommunity(mode):
    g = O.Graph.from_edges(4, *weighted([(0, 1, 10.0), (0, 3, 100.0), (1, 3, 100.0), (1, 2, 1.0)]))
    s, r = O.inc_refinement(g, [0, 0, 0, 1], [0, 1, 2, 3], [1, 1, 1, 1], 1.0, mode)
    assert s[2] == 2


# --- aggregation self-loop transfer (hit_leiden.rs:2120-2178) ---------------
def test_aggregation_self_loop_transfer():
    g = O.Graph.from_edges(3, *weighted([(0, 0, 5.0), (0, 1, 1.0), (1, 2, 1.0)]))
    (u, v, w), nsp, nn = O.inc_aggregation(g, [], [], [], [0, 1, 2], [1, 1, 2], [1, 0, 0])
    sl0 = sum(wi for ui, vi, wi in zip(u, v, w) if ui == 0 and vi == 0)
    sl1 = sum(wi for ui, vi, wi in zip(u, v, w) if ui == 1 and vi == 1)
    assert sl0 < -1e-9 and sl1 > 1e-9
    # Reference quirk: both CSR copies are summed, so 2w moves (:1682-1692).
    assert sl0 == -10.0


def test_aggregation_self_loop_transfer_edge_weight_option():
    g = O.Graph.from_edges(3, *weighted([(0, 0, 5.0), (0, 1, 1.0), (1, 2, 1.0)]))
    (u, v, w), _, _ = O.inc_aggregation(g, [], [], [], [0, 1, 2], [1, 1, 2], [1, 0, 0],
                                        flags=O.FLAG_EDGE_WEIGHT_LOOPS)
    sl1 = sum(wi for ui, vi, wi in zip(u, v, w) if ui == 1 and vi == 1)
    # w(0,0)=5 moves plus edge (0,1) becomes internal to sub-community 1.
    assert sl1 == 6.0


# --- modularity KATs (hit_leiden.rs:2185-2272) ------------------------------
def test_modularity_single_community_triangle():
    assert abs(O.modularity_edges(3, *unit([(0, 1), (1, 2), (0, 2)]), [0, 0, 0])) < 1e-9


def test_modularity_all_singletons_triangle():
    q = O.modularity_edges(3, *unit([(0, 1), (1, 2), (0, 2)]), [0, 1, 2])
    assert abs(q - (-1.0 / 3.0)) < 1e-9


def test_modularity_two_cliques_optimal():
    e = [(0, 1), (1, 2), (0, 2), (3, 4), (4, 5), (3, 5)]
    assert abs(O.modularity_edges(6, *unit(e), [0, 0, 0, 1, 1, 1]) - 0.5) < 1e-9


def test_modularity_empty_graph():
    assert abs(O.modularity_edges(3, [], [], [], [0, 1, 2])) < 1e-9


def test_modularity_weighted_edges():
    src, dst, w = weighted([(0, 1, 5.0)])
    assert abs(O.modularity_edges(2, src, dst, w, [0, 0])) < 1e-9
    assert abs(O.modularity_edges(2, src, dst, w, [0, 1]) - (-0.5)) < 1e-9


def test_modularity_csr_matches_edge_list_form():
    rng = np.random.default_rng(3)
    n = 50
    src = rng.integers(0, n, 200)
    dst = rng.integers(0, n, 200)
    w = rng.integers(1, 4, 200).astype(float)
    part = rng.integers(0, 7, n)
    g = O.Graph.from_edges(n, src, dst, w)
    q1 = O.modularity_edges(n, src, dst, w, part)
    q2 = O.modularity_csr(g, part)
    assert abs(q1 - q2) <= 1e-12 * max(1.0, abs(q1))


# --- gain sign (hit_leiden.rs:2280-2348) ------------------------------------
@pytest.mark.parametrize("mode", MODES)
def test_modularity_gain_positive_for_natural_move(mode):
    g = O.Graph.from_edges(5, *weighted([(0, 1, 10.0), (1, 2, 0.1), (2, 3, 10.0), (2, 4, 10.0),
                                         (3, 4, 10.0)]))
    f, ch, k, it = O.inc_movement(g, [], [], [], [0, 0, 0, 1, 1], [0, 1, 2, 3, 4], 1.0, mode)
    assert f[2] == f[3] and ch[2]


@pytest.mark.parametrize("mode", MODES)
def test_modularity_gain_no_move_for_well_connected(mode):
    g = O.Graph.from_edges(4, *unit([(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]))
    f, ch, k, it = O.inc_movement(g, [], [], [], [0, 0, 0, 0], [0, 1, 2, 3], 1.0, mode)
    assert not ch.any()


# --- multilevel run() (hit_leiden.rs:2354-2446) ------------------------------
def test_multilevel_leiden_two_cliques():
    e = [(0, 1), (1, 2), (0, 2), (3, 4), (4, 5), (3, 5), (2, 3)]
    part, q, lv = O.run(6, *unit(e))
    assert lv >= 1
    assert len(set(part.tolist())) == 2
    assert part[0] == part[1] == part[2] and part[3] == part[4] == part[5] and part[0] != part[3]


def test_multilevel_leiden_single_node():
    part, q, lv = O.run(1, [], [])
    assert part.tolist() == [0] and lv >= 1


def test_multilevel_leiden_disconnected_components():
    part, q, lv = O.run(4, [], [])
    assert len(set(part.tolist())) == 4


# --- canonicalize (hit_leiden.rs:2448-2461) ---------------------------------
def test_canonicalize_community_ids():
    assert O.canonicalize([5, 5, 3, 3, 7]).tolist() == [0, 0, 1, 1, 2]
    assert O.canonicalize([0, 0, 1, 1, 2]).tolist() == [0, 0, 1, 1, 2]


# --- A/K seeding (hit_leiden.rs:2468-2603) -----------------------------------
@pytest.mark.parametrize("mode", MODES)
def test_inc_movement_cross_community_insertion_activates(mode):
    g = O.Graph.from_edges(3, *weighted([(0, 1, 1.0), (1, 2, 10.0)]))
    f, ch, k, it = O.inc_movement(g, *weighted([(1, 2, 10.0)]), [0, 0, 1], [0, 0, 1], 1.0, mode)
    if mode == O.MODE_DETERMINISTIC:
        assert f[1] == f[2]
    else:
        assert len(set(f.tolist())) <= 3


@pytest.mark.parametrize("mode", MODES)
def test_inc_movement_intra_community_deletion_activates(mode):
    g = O.Graph.from_edges(4, *weighted([(0, 1, 10.0), (2, 3, 10.0)]))
    f, ch, k, it = O.inc_movement(g, *weighted([(0, 2, -1.0)]), [0, 0, 0, 1], [0, 1, 2, 3], 1.0,
                                  mode)
    assert f[2] == f[3] and ch[2]


@pytest.mark.parametrize("mode", MODES)
def test_inc_movement_same_subcommunity_edge_tracks_k(mode):
    g = O.Graph.from_edges(3, *unit([(0, 1), (1, 2)]))
    f, ch, k, it = O.inc_movement(g, *weighted([(0, 1, -1.0)]), [0, 0, 0], [0, 0, 2], 1.0, mode)
    assert k[0] and k[1]


@pytest.mark.parametrize("mode", MODES)
def test_inc_movement_neighbor_requeuing(mode):
    g = O.Graph.from_edges(4, *weighted([(0, 1, 10.0), (1, 2, 0.1), (2, 3, 10.0)]))
    f, ch, k, it = O.inc_movement(g, [], [], [], [0, 0, 0, 1], [0, 1, 2, 3], 1.0, mode)
    if mode == O.MODE_DETERMINISTIC:
        assert f[2] == f[3] and f[0] == f[1] and f[0] != f[2]
    else:
        assert f[0] == f[1] and len(set(f.tolist())) == 2


# --- CC split (hit_leiden.rs:2676-2758) -------------------------------------
@pytest.mark.parametrize("mode", MODES)
def test_refinement_splits_disconnected_subcommunity(mode):
    g = O.Graph.from_edges(4, *unit([(0, 1), (2, 3)]))
    s, r = O.inc_refinement(g, [0, 0, 0, 0], [0, 0, 0, 0], [1, 1, 1, 1], 1.0, mode)
    assert s[0] == s[1] and s[2] == s[3] and s[0] != s[2]


@pytest.mark.parametrize("mode", MODES)
def test_refinement_largest_component_retains_id(mode):
    g = O.Graph.from_edges(5, *unit([(0, 1), (1, 2), (3, 4)]))
    s, r = O.inc_refinement(g, [0] * 5, [0] * 5, [1] * 5, 1.0, mode)
    assert s[0] == 0 and s[1] == 0 and s[2] == 0 and s[3] != 0 and s[3] == s[4]


def test_refinement_equal_components_keep_last():
    # Rust max_by_key keeps the last maximum (hit_leiden.rs:1317-1322):
    # components {0,1} and {2,3} are equal, so {2,3} keeps the id.
    g = O.Graph.from_edges(4, *unit([(0, 1), (2, 3)]))
    s, r = O.inc_refinement(g, [0] * 4, [0] * 4, [1] * 4, 1.0, O.MODE_THROUGHPUT)
    assert s[2] == 0 and s[3] == 0 and s[0] == 1 and s[1] == 1
    assert r.tolist() == [True, True, False, False]


# --- singleton merge (hit_leiden.rs:2760-2794) ------------------------------
@pytest.mark.parametrize("mode", MODES)
def test_refinement_singleton_merge_positive_gain(mode):
    g = O.Graph.from_edges(3, *weighted([(0, 1, 10.0), (1, 2, 10.0)]))
    s, r = O.inc_refinement(g, [0, 0, 0], [0, 1, 2], [1, 1, 1], 1.0, mode)
    assert len(set(s.tolist())) < 3


# --- affected-only (hit_leiden.rs:2796-2838) --------------------------------
@pytest.mark.parametrize("mode", MODES)
def test_refinement_only_processes_affected_subcommunities(mode):
    g = O.Graph.from_edges(4, *unit([(0, 1), (2, 3)]))
    s, r = O.inc_refinement(g, [0, 0, 1, 1], [0, 0, 2, 2], [0, 0, 1, 1], 1.0, mode)
    assert s[0] == 0 and s[1] == 0


# --- inc-aggregation (hit_leiden.rs:2840-2993) -------------------------------
def test_aggregation_maps_delta_via_s_pre_not_s_cur():
    g = O.Graph.from_edges(4, *unit([(0, 1), (1, 2), (2, 3)]))
    (u, v, w), _, _ = O.inc_aggregation(g, *weighted([(0, 2, 5.0)]), [0, 0, 2, 2], [0, 0, 0, 2],
                                        [0, 0, 0, 0])
    inter = sum(wi for ui, vi, wi in zip(u, v, w) if min(ui, vi) == 0 and max(ui, vi) == 2)
    assert abs(inter - 5.0) < 1e-9


def test_aggregation_compress_sums_duplicates():
    g = O.Graph.from_edges(4, *unit([(0, 1), (2, 3)]))
    (u, v, w), _, _ = O.inc_aggregation(g, *weighted([(0, 2, 3.0), (1, 3, 2.0)]), [0, 0, 1, 1],
                                        [0, 0, 1, 1], [0, 0, 0, 0])
    tot = sum(wi for ui, vi, wi in zip(u, v, w) if {ui, vi} == {0, 1})
    assert abs(tot - 5.0) < 1e-9 and len(u) == 1


def test_aggregation_removes_zero_weight_edges():
    g = O.Graph.from_edges(4, *unit([(0, 1), (2, 3)]))
    (u, v, w), _, _ = O.inc_aggregation(g, *weighted([(0, 2, 3.0), (0, 3, -3.0)]), [0, 0, 1, 1],
                                        [0, 0, 1, 1], [0, 0, 0, 0])
    assert len(u) == 0


def test_aggregation_updates_s_pre_for_refined_nodes():
    g = O.Graph.from_edges(3, *unit([(0, 1), (1, 2)]))
    _, nsp, nn = O.inc_aggregation(g, [], [], [], [0, 1, 2], [0, 1, 1], [0, 0, 1])
    assert nsp.tolist() == [0, 1, 1] and nn == 3


# --- def-update (hit_leiden.rs:2995-3098) -----------------------------------
def test_def_update_propagates_community_assignments():
    f = [[0, 0, 1, 1], [1, 1]]
    s = [[0, 0, 1, 1], [0, 1]]
    ch = [[0, 0, 0, 0], [1, 0]]
    f2, c2 = O.def_update(f, s, ch)
    assert f2[0][0] == 1 and f2[0][1] == 1


def test_def_update_propagates_changed_nodes_downward():
    f = [[0, 0, 1, 1], [0, 1]]
    s = [[0, 0, 1, 1], [0, 1]]
    ch = [[0, 0, 0, 0], [0, 1]]
    f2, c2 = O.def_update(f, s, ch)
    assert c2[0].tolist() == [False, False, True, True]


def test_def_update_skips_boundary_levels():
    f2, c2 = O.def_update([[0, 1, 2]], [[0, 1, 2]], [[1, 0, 0]])
    assert f2[0].tolist() == [0, 1, 2]


# --- end-to-end incremental (hit_leiden.rs:3104-3251) ------------------------
@pytest.mark.parametrize("mode", MODES)
def test_hit_leiden_initial_run_finds_communities(mode):
    e = [(0, 1), (1, 2), (0, 2), (3, 4), (4, 5), (3, 5), (2, 3)]
    st = O.State(6, mode=mode)
    st.push_empty_graph()
    st.hit_leiden(*unit(e))
    # node_to_comm is g¹, which stays the identity at one level: ≥ 2 communities.
    assert len(set(st.get_map(0, O.MAP_NODE_TO_COMM).tolist())) >= 2


@pytest.mark.parametrize("mode", MODES)
def test_hit_leiden_incremental_adapts_to_new_edge(mode):
    e = [(0, 1, 10.0), (1, 2, 10.0), (0, 2, 10.0), (3, 4, 10.0), (4, 5, 10.0), (3, 5, 10.0),
         (2, 3, 0.1)]
    st = O.State(6, mode=mode)
    st.push_empty_graph()
    st.hit_leiden(*weighted(e))
    c0 = len(set(st.get_map(0, O.MAP_NODE_TO_COMM).tolist()))
    st.hit_leiden(*weighted([(0, 3, 100.0), (1, 4, 100.0)]))
    assert len(set(st.get_map(0, O.MAP_NODE_TO_COMM).tolist())) <= c0


@pytest.mark.parametrize("mode", MODES)
def test_hit_leiden_incremental_adapts_to_edge_removal(mode):
    st = O.State(4, mode=mode)
    st.push_empty_graph()
    st.hit_leiden(*unit([(0, 1), (1, 2), (2, 3)]))
    st.hit_leiden(*weighted([(1, 2, -1.0)]))
    assert 2 not in [n for n, _ in st.graph(0).neighbors(1)]


@pytest.mark.parametrize("mode", MODES)
def test_hit_leiden_delta_g_flows_between_levels(mode):
    e = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3), (4, 5), (4, 6), (4, 7), (5, 6), (5, 7),
         (6, 7), (3, 4)]
    st = O.State(8, mode=mode)
    st.push_empty_graph()
    st.hit_leiden(*unit(e))
    st.hit_leiden(*weighted([(0, 4, 50.0), (1, 5, 50.0)]))
    assert len(set(st.get_map(0, O.MAP_NODE_TO_COMM).tolist())) >= 1


# --- idempotence (hit_leiden.rs:3361-3400) -----------------------------------
@pytest.mark.parametrize("mode", MODES)
def test_movement_idempotent_on_stable_partition(mode):
    g = O.Graph.from_edges(6, *unit([(0, 1), (1, 2), (0, 2), (3, 4), (4, 5), (3, 5), (2, 3)]))
    s = [0, 0, 0, 1, 1, 1]
    f1, *_ = O.inc_movement(g, [], [], [], [0, 0, 0, 1, 1, 1], s, 1.0, mode)
    f2, *_ = O.inc_movement(g, [], [], [], f1, s, 1.0, mode)
    assert np.array_equal(f1, f2)


# --- decoupled selection (throughput.rs:369-400) -----------------------------
def test_decoupling_blocks_reverse_conflicts():
    sel = O.select_decoupled([1, 2, 3], [10, 20, 30], [20, 10, 40], [10.0, 9.0, 8.0])
    assert sel.tolist() == [1, 3]


def test_decoupling_allows_emit_and_accept_consistency():
    sel = O.select_decoupled([10, 11, 12, 13], [1, 1, 4, 2], [2, 3, 2, 5], [10.0, 9.0, 8.0, 7.0])
    assert sel.tolist() == [10, 11, 12]


def test_decoupling_tie_breaks_by_node_ascending():
    sel = O.select_decoupled([7, 3], [1, 2], [2, 1], [5.0, 5.0])
    assert sel.tolist() == [3]


# --- empty-community id and the fixed-snapshot decision -----------------------
def test_move_eval_empty_community_id_is_n_plus_v():
    g = O.Graph.from_edges(3, *weighted([(0, 1, 10.0), (0, 2, 0.5)]))
    k = g.degrees()
    d = np.zeros(6)
    d[0] = k.sum()
    to, gain = O.move_eval(g, [0, 0, 0], d, k, k.sum(), 3.0, [2])
    assert to[0] == 3 + 2 and gain[0] > 0


def test_move_eval_first_encountered_wins_ties():
    # Node 0 sees communities 5 and 4 with identical weight and degree: the one
    # met first in CSR order (neighbour 1 → community 5) wins the strict '>'.
    g = O.Graph.from_edges(3, *unit([(0, 1), (0, 2)]))
    f = [0, 5, 4]
    k = g.degrees()
    d = np.zeros(6)
    for v in range(3):
        d[f[v]] += k[v]
    to, gain = O.move_eval(g, f, d, k, k.sum(), 1.0, [0])
    assert to[0] == 5


def test_tree_sum_is_exact_for_integers():
    x = np.arange(5000, dtype=np.float64)
    assert O.tree_sum(x) == float(x.sum())


def test_results_do_not_depend_on_host_threads():
    # The throughput mode's snapshot evaluations run on host threads; the
    # state after a bootstrap and batches must not depend on how many.
    import importlib
    W = importlib.import_module("hit-leiden_b200.workloads")
    n, s, d, w, _ = W.planted(3000, 8.0, 0.25, 9, comm_min=5, comm_max=80, weights=(0.5, 2.0))
    states = []
    for threads in (1, 8):
        O.set_num_threads(threads)
        st = O.State(n, mode=O.MODE_THROUGHPUT)
        st.bootstrap(s, d, w, max_levels=6)
        store = W.EdgeStore(n, s, d, w)
        for b in range(3):
            u, v, ww = W.mixed_batch(store, 300, 0.9, 50 + b, weights=(0.5, 2.0))
            st.hit_leiden(u, v, ww)
        states.append(st)
    O.set_num_threads(0)
    a, b = states
    assert a.levels == b.levels
    for p in range(a.levels):
        for which in (O.MAP_F, O.MAP_G, O.MAP_S_PRE, O.MAP_S_CUR):
            assert np.array_equal(a.get_map(p, which), b.get_map(p, which))


# --- run() integration and property tests (tests/integration/*.rs, ----------
# --- tests/property/test_partition_invariants.rs) ---------------------------

def test_run_connected_graph_not_all_singletons():
    # test_connected_graph_not_all_singletons.rs:21-49: two triangles and a
    # 0.05 bridge merge at least one pair
    src, dst, w = weighted([(0, 1, 1.0), (1, 2, 1.0), (2, 0, 1.0), (3, 4, 1.0), (4, 5, 1.0),
                            (5, 3, 1.0), (2, 3, 0.05)])
    part, _, _ = O.run(6, src, dst, w)
    assert len(set(part.tolist())) < 6
    st = O.State(6, mode=O.MODE_THROUGHPUT)
    st.bootstrap(src, dst, w, max_levels=10)
    assert len(set(st.get_map(0, O.MAP_F).tolist())) < 6


def test_run_deterministic_replay_identity():
    # test_deterministic_identity.rs:19-30: two runs on the same input agree
    src, dst, w = unit([(0, 1), (2, 3)])
    a = O.run(4, src, dst, w)
    b = O.run(4, src, dst, w)
    assert np.array_equal(a[0], b[0]) and a[1] == b[1]


@pytest.mark.parametrize("n", [0, 1, 2, 7, 31, 49])
def test_run_partition_length_matches_node_count(n):
    # test_partition_invariants.rs:20-32: isolated nodes, node_count in 0..50
    part, q, _ = O.run(n, [], [], [])
    assert len(part) == n and q == 0.0
    if n:
        st = O.State(n, mode=O.MODE_THROUGHPUT)
        st.bootstrap([], [], [], max_levels=10)
        assert len(st.get_map(0, O.MAP_F)) == n


def test_deterministic_empty_moves_take_successive_ids():
    """Deterministic movement (hit_leiden.rs:1150-1173): each move to the
    empty community takes community_degrees.len(), and the array grows by
    one, so a second empty move gets the next id.  At gamma = 3 on
    0-1 (10), 0-2 (0.5), node 0 leaves for id 3, then node 1 (whose only
    neighbour is now in 3, at a negative gain) leaves for id 4."""
    g = O.Graph.from_edges(3, np.array([0, 0], np.uint32), np.array([1, 2], np.uint32),
                           np.array([10.0, 0.5]))
    f, changed, _, it = O.inc_movement(g, [], [], None, [0, 0, 0], [0, 0, 0], 3.0,
                                       O.MODE_DETERMINISTIC)
    assert f.tolist() == [3, 4, 0] and changed.tolist() == [True, True, False] and it == 1
