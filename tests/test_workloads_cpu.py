"""The seeded synthetic inputs that stand in for the reference's datasets
have the documented shapes: sizes, degrees, weights, mixing and the batch
mixes (hit-leiden_b200/workloads.py).  Checked on the CPU at the stated sizes,
or at a reduced vertex count where generation at full size would take long."""
import importlib

import numpy as np
import pytest

W = importlib.import_module("hit-leiden_b200.workloads")


def _canonical(n, s, d):
    assert len(s) == len(d)
    assert np.all(s < d), "edges are stored once, src < dst, no self-loops"
    key = s.astype(np.int64) * n + d.astype(np.int64)
    assert len(np.unique(key)) == len(key), "no duplicate edges"


def test_config1_shape():
    # ca-HepTh's shape: 9,877 vertices, ~21.8k unit edges, mean degree ~4.4
    n, s, d, w = W.config1(0)
    assert n == 9877
    _canonical(n, s, d)
    assert 19_000 <= len(s) <= 24_500
    assert 3.8 <= 2 * len(s) / n <= 5.0
    assert np.all(w == 1.0)
    # target degrees are capped at 65 (ca-HepTh's maximum); wedge closure for
    # the clustering adds edges on top of them
    deg = np.bincount(np.concatenate([s, d]), minlength=n)
    assert 50 <= deg.max() <= 2 * 65


def test_config2_shape_reduced():
    # the 1M-vertex configuration's parameters at 200k vertices: mean degree
    # 40, degrees capped at 2000, f64 weights U[0.5, 2]
    n, s, d, w = W.config2(0, n=200_000)
    _canonical(n, s, d)
    mean = 2 * len(s) / n
    assert 36.0 <= mean <= 44.0, mean
    deg = np.bincount(np.concatenate([s, d]), minlength=n)
    assert deg.max() <= 2000
    assert w.min() >= 0.5 and w.max() <= 2.0 and len(np.unique(w)) > len(w) // 2


@pytest.mark.parametrize("mu", [0.15, 0.3])
def test_planted_mixing_and_community_sizes(mu):
    n, s, d, w, comm = W.planted(50_000, 20.0, mu, 1, comm_min=50, comm_max=5000)
    _canonical(n, s, d)
    cross = float(np.mean(comm[s] != comm[d]))
    assert abs(cross - mu) < 0.05, cross
    sizes = np.bincount(comm)
    sizes = sizes[sizes > 0]
    assert sizes.min() >= 50 and sizes.max() <= 5000


def test_config4_shape():
    gs = W.config4(0, count=6)
    assert len(gs) == 6
    for n, s, d, w in gs:
        assert 1000 <= n <= 200_000
        _canonical(n, s, d)
        assert 2.0 <= 2 * len(s) / n <= 34.0
        assert np.all(w == 1.0)


def test_config5_shape_scaled():
    gs = W.config5(0, count=3, scale=0.01)
    for n, s, d, w in gs:
        assert 1000 <= n <= 50_000
        _canonical(n, s, d)
        assert 8.0 <= 2 * len(s) / n <= 20.0


def test_mixed_batch_inserts_and_exact_deletes():
    n, s, d, w, _ = W.planted(3000, 8.0, 0.2, 2, weights=(0.5, 2.0))
    store = W.EdgeStore(n, s, d, w)
    before = {(a, b): x for a, b, x in zip(s.tolist(), d.tolist(), w.tolist())}
    u, v, x = W.mixed_batch(store, 1000, 0.9, 5, weights=(0.5, 2.0))
    assert len(u) == 1000 and np.all(u != v)
    dels = x < 0
    assert int(dels.sum()) == 100
    for a, b, y in zip(u[dels].tolist(), v[dels].tolist(), x[dels].tolist()):
        key = (min(a, b), max(a, b))
        assert before[key] == -y, "a delete removes the edge's whole weight"
    assert np.all((x[~dels] >= 0.5) & (x[~dels] <= 2.0))


def test_uniform_inserts_are_new_unit_edges():
    n, s, d, w = W.config1(1)
    ex = set(zip(s.tolist(), d.tolist()))
    u, v, x = W.uniform_inserts(n, 1000, 3, ex)
    assert len(u) == 1000 and np.all(u != v) and np.all(x == 1.0)
    keys = {(min(a, b), max(a, b)) for a, b in zip(u.tolist(), v.tolist())}
    assert len(keys) == 1000 and not keys & ex


def test_rmat_symmetrised_and_deduplicated():
    pytest.importorskip("torch")
    n, bs, bd = W.rmat_torch(10, 16, 0, device="cpu")
    s = bs.numpy().view(np.uint32)
    d = bd.numpy().view(np.uint32)
    assert n == 1024
    _canonical(n, s, d)
    assert 0 < len(s) <= 16 * 1024
    deg = np.bincount(np.concatenate([s, d]), minlength=n)
    assert deg[:16].mean() > 4 * deg.mean(), "R-MAT skews degree to low ids"


def test_fast_batch_shape():
    n, s, d, w = W.config1(0)
    u, v, x = W.fast_batch(n, s, d, 500, 0.85, 9)
    assert len(u) == 500 and np.all(u != v)
    assert int((x > 0).sum()) == 425 and np.all(np.abs(x) == 1.0)
