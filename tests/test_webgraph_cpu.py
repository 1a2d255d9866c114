"""The BV (WebGraph) loader in the reference's conventions
(src/main.rs:189-230): a hand-assembled bit stream decodes to its lists, the
encoder and decoder round-trip graphs that use references, copy blocks,
intervals and residuals, and load_webgraph keeps src < dst and skips
self-loops."""
import importlib

import numpy as np
import pytest

WG = importlib.import_module("hit-leiden_b200.webgraph")


def _write_raw(tmp_path, bits, props):
    bits = bits + "0" * (-len(bits) % 8)
    data = bytes(int(bits[i:i + 8], 2) for i in range(0, len(bits), 8))
    base = str(tmp_path / "kat")
    open(base + ".graph", "wb").write(data)
    open(base + ".properties", "w").write("\n".join(f"{k}={v}" for k, v in props.items()) + "\n")
    return base


def test_hand_assembled_stream():
    # 3 nodes {0: [1, 2], 1: [0], 2: [0, 1]}, no references, no intervals,
    # zeta_3 residuals.  Node 0: gamma(2)=011, residual int2nat(1-0)=2 ->
    # zeta_3 1011, gap 0 -> 100.  Node 1: gamma(1)=010, int2nat(0-1)=1 ->
    # 1010.  Node 2: 011, int2nat(0-2)=3 -> 1100, gap 0 -> 100.
    import tempfile
    import pathlib
    bits = "011" "1011" "100" "010" "1010" "011" "1100" "100"
    with tempfile.TemporaryDirectory() as td:
        base = _write_raw(pathlib.Path(td), bits,
                          {"nodes": 3, "arcs": 5, "windowsize": 0, "minintervallength": 0,
                           "zetak": 3, "compressionflags": ""})
        succ = WG.read_bvgraph(base)
    assert [s.tolist() for s in succ] == [[1, 2], [0], [0, 1]]


def _local_graph(rng, n, deg):
    """Successor lists with locality: runs of consecutive ids (intervals) and
    lists shared with earlier nodes (references, copy blocks)."""
    succ = []
    for x in range(n):
        lst = set()
        if x and rng.random() < 0.5:
            prev = succ[x - int(rng.integers(1, min(x, 7) + 1))]
            lst.update(v for v in prev if rng.random() < 0.8)
        if rng.random() < 0.5:
            a = int(rng.integers(0, n))
            lst.update(range(a, min(n, a + int(rng.integers(4, 12)))))
        lst.update(int(v) for v in rng.integers(0, n, int(rng.integers(0, deg))))
        succ.append(sorted(lst))
    return succ


@pytest.mark.parametrize("window,min_interval,k,flags", [
    (7, 4, 3, ""), (3, 2, 2, ""), (0, 0, 3, ""), (7, 4, 3, "RESIDUALS_GAMMA|OUTDEGREES_DELTA")])
def test_round_trip(tmp_path, window, min_interval, k, flags):
    rng = np.random.default_rng(window * 10 + min_interval)
    succ = _local_graph(rng, 600, 12)
    base = str(tmp_path / "g")
    used = WG.write_bvgraph(base, succ, window=window, min_interval=min_interval, zeta_k=k,
                            flags=flags)
    if window:
        assert used["references"] > 50
    if min_interval:
        assert used["intervals"] > 50
    got = WG.read_bvgraph(base)
    assert [g.tolist() for g in got] == succ


def test_load_webgraph_reference_conventions(tmp_path):
    # symmetric listing with a self-loop on node 2 and an isolated node 4
    succ = [[1, 3], [0, 2], [1, 2, 3], [0, 2], []]
    base = str(tmp_path / "sym")
    WG.write_bvgraph(base, succ)
    e = WG.load_webgraph(base)
    assert e.node_count == 5 and e.self_loops_skipped == 1
    assert sorted(zip(e.src.tolist(), e.dst.tolist())) == [(0, 1), (0, 3), (1, 2), (2, 3)]
    assert np.all(e.w == 1.0) and e.dataset_id == "sym"


def test_corrupt_stream_is_rejected(tmp_path):
    base = str(tmp_path / "bad")
    WG.write_bvgraph(base, [[1], [0]])
    open(base + ".properties", "a").write("")
    props = WG.read_properties(base + ".properties")
    props["nodes"] = "40"  # more nodes than the stream holds
    open(base + ".properties", "w").write("\n".join(f"{k}={v}" for k, v in props.items()))
    with pytest.raises(ValueError):
        WG.read_bvgraph(base)
