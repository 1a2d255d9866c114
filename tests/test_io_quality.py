"""Host-side loaders, batch schedules and the partition quality report
(hit-leiden_b200/io.py), checked on the CPU against the reference's tests and
against independent implementations."""
import importlib
import math

import numpy as np
import pytest

IO = importlib.import_module("hit-leiden_b200.io")


def test_parse_skips_comments_and_self_loops():
    e = IO.parse_edge_list("# comment\n% other\n\n0 1\n1 1\n2 0 2.5\n3,4,0.5\n")
    assert e.src.tolist() == [0, 0, 3] and e.dst.tolist() == [1, 2, 4]
    assert e.w.tolist() == [1.0, 2.5, 0.5]
    assert e.node_count == 5 and e.self_loops_skipped == 1


def test_parse_symmetric_keeps_one_direction():
    # webgraph-style listing with both directions (main.rs:189-230)
    e = IO.parse_edge_list("0 1\n1 0\n1 2\n2 1\n2 2\n", symmetric=True)
    assert list(zip(e.src.tolist(), e.dst.tolist())) == [(0, 1), (1, 2)]
    assert e.self_loops_skipped == 1


def test_parse_rejects_bad_lines_and_small_node_count():
    with pytest.raises(ValueError):
        IO.parse_edge_list("0\n")
    with pytest.raises(ValueError):
        IO.parse_edge_list("0 5\n", node_count=3)
    assert IO.parse_edge_list("0 5\n", node_count=10).node_count == 10


def test_load_edge_list_file(tmp_path):
    p = tmp_path / "toy.txt"
    p.write_text("0 1\n1 2\n")
    e = IO.load_edge_list(str(p))
    assert e.dataset_id == "toy" and len(e) == 2


def _edges(m, n=50, seed=0):
    rng = np.random.default_rng(seed)
    s = rng.integers(0, n, m).astype(np.uint32)
    d = ((s + 1 + rng.integers(0, n - 1, m)) % n).astype(np.uint32)
    return IO.EdgeList("t", n, np.minimum(s, d), np.maximum(s, d), np.ones(m))


def test_paper_split_shape_matches_reference():
    # dynamic_graph.rs:139-155: 100 edges, ratio 0.8, batch 5, 4 rounds
    sp = IO.paper_split(_edges(100), 0.8, 5, 4, 42)
    assert len(sp.initial) == 80
    assert [len(u) for u in sp.updates] == [85, 90, 95, 100]
    assert all(len(d) == 5 for d in sp.deltas)
    assert sp.batch_size == 5 and sp.rounds == 4
    # rounds capped by the edges left
    assert IO.paper_split(_edges(100), 0.8, 5, 10, 1).rounds == 4


def test_cumulative_batches():
    b = IO.cumulative_batches(_edges(23), 10)
    assert [len(x) for x in b] == [10, 20, 23]


def test_nmi_against_independent_implementation():
    sk = pytest.importorskip("sklearn.metrics")
    rng = np.random.default_rng(3)
    for _ in range(5):
        a = rng.integers(0, 7, 500)
        b = np.where(rng.random(500) < 0.7, a, rng.integers(0, 9, 500))
        r = IO.compare_partitions(a, b)
        ref = sk.normalized_mutual_info_score(a, b, average_method="geometric")
        assert abs(r.nmi - ref) < 1e-12


def test_identical_and_relabelled_partitions():
    a = np.array([0, 0, 1, 1, 2, 2, 2])
    r = IO.compare_partitions(a, a)
    assert math.isclose(r.nmi, 1.0) and r.purity_a_to_b == 1.0 and r.largest_jaccard == 1.0
    r = IO.compare_partitions(a, 10 - a)
    assert math.isclose(r.nmi, 1.0) and r.largest_jaccard == 1.0


def test_purity_and_largest_jaccard_by_hand():
    a = [0, 0, 0, 1, 1, 2]
    b = [5, 5, 6, 6, 6, 6]
    r = IO.compare_partitions(a, b)
    # a -> b: community 0 best 2, 1 best 2, 2 best 1 => 5/6; b -> a: 5 best 2, 6 best 2 => 4/6
    assert math.isclose(r.purity_a_to_b, 5 / 6) and math.isclose(r.purity_b_to_a, 4 / 6)
    # largest: a -> id 0 (size 3), b -> id 6 (size 4); intersection 1, union 6
    assert math.isclose(r.largest_jaccard, 1 / 6)
    assert (r.communities_a, r.communities_b, r.largest_a, r.largest_b) == (3, 2, 3, 4)


def test_largest_community_tie_takes_smallest_id():
    assert IO.largest_community([4, 4, 2, 2, 9]) == (2, 2)


def test_single_community_partition_has_zero_nmi():
    r = IO.compare_partitions([0, 0, 0], [1, 2, 3])
    assert r.nmi == 0.0
