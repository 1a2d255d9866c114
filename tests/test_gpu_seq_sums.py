"""The ordered f64 sums on the GPU, through hl_dbg_seq_sums: every segment's
left-to-right fold, bit for bit, by the library's own pair of kernels (segments
below 512 terms one addition after another, longer ones in runs of same-binade
terms) and by each fold alone.  These are the sums behind the row sums in CSR
order (hit_leiden.rs:1063), the community degrees and the aggregation's
per-super-edge weights; the row sums of a graph with hub rows are also checked
against the oracle's degrees.

Tolerance: bit-exact (NaN matches NaN)."""
import ctypes as C
import importlib
import math

import numpy as np
import pytest

from fold_cases import KINDS, grid_ties, seq_fold, terms
from oracle import oracle as O

pytestmark = pytest.mark.gpu

L = importlib.import_module("hit-leiden_b200._lib")

LENGTHS = [0, 1, 2, 31, 32, 33, 127, 128, 129, 255, 256, 511, 512, 513, 1000, 4096, 20000, 70000]


def _gpu(segs, init, path):
    off = np.zeros(len(segs) + 1, np.uint64)
    off[1:] = np.cumsum([len(s) for s in segs])
    x = np.concatenate([np.asarray(s, np.float64) for s in segs] + [np.zeros(1)])
    out = np.zeros(max(1, len(segs)))
    L.check(L.lib.hl_dbg_seq_sums(0, len(segs), L.ptr(off), L.ptr(x), init, path, L.ptr(out)))
    return out[:len(segs)]


def _same(a, b):
    return a.view(np.uint64) == b.view(np.uint64) or (math.isnan(a) and math.isnan(b))


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("path", [0, 1, 2])
def test_seq_sums_bit_exact(kind, path):
    rng = np.random.default_rng(KINDS.index(kind) + 17 * path)
    segs = [terms(kind, n, rng) for n in LENGTHS]
    for init in (0.0, float(2 ** 52 - 7), -3.5):
        got = _gpu(segs, init, path)
        for i, s in enumerate(segs):
            want = np.float64(seq_fold(s, init))
            assert _same(got[i], want), (kind, path, init, len(s), got[i], want)


@pytest.mark.parametrize("path", [0, 1])
def test_seq_sums_exact_ties_on_the_grid(path):
    # terms on the start's grid, a quarter of them exact ties, in long
    # segments: the run fold must leave each tie to an ordinary addition
    rng = np.random.default_rng(3 + path)
    for k in (-20, -1, 0, 7, 30):
        acc0, xs = grid_ties(rng, 3000, k)
        for a0 in (acc0, -acc0):
            got = _gpu([xs, xs[:600], xs[:513]], a0, path)
            for g, s in zip(got, (xs, xs[:600], xs[:513])):
                assert _same(g, np.float64(seq_fold(s, a0)))


def test_seq_sums_many_long_segments():
    # more long segments than the run kernel has warps, of mixed lengths
    rng = np.random.default_rng(8)
    segs = [rng.uniform(0.5, 2.0, int(n)) for n in rng.integers(400, 1500, 3000)]
    got = _gpu(segs, 0.0, 0)
    for g, s in zip(got, segs):
        assert _same(g, np.float64(seq_fold(s, 0.0)))


def test_row_sums_of_hub_rows_match_oracle_degrees():
    rng = np.random.default_rng(21)
    n = 30000
    src = [rng.integers(0, n, 60000)]
    dst = [rng.integers(0, n, 60000)]
    for hub, deg in ((0, 600), (1, 5000), (2, 25000)):
        src.append(np.full(deg, hub))
        dst.append(rng.choice(np.arange(3, n), deg, replace=False))
    s = np.concatenate(src).astype(np.uint32)
    d = np.concatenate(dst).astype(np.uint32)
    w = rng.uniform(0.5, 2.0, len(s))
    g = O.Graph.from_edges(n, s, d, w)
    off, col, ww = g.csr()
    deg = np.diff(off)
    assert deg.max() >= 25000
    got = _gpu([ww[off[v]:off[v + 1]] for v in range(n)], 0.0, 0)
    want = g.degrees()
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
