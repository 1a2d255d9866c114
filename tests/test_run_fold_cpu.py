"""The run fold behind the long ordered f64 sums (row sums in CSR order,
hit_leiden.rs:1063; community degrees; the aggregation's per-super-edge sums),
restated here lane by lane in numpy and checked bitwise against a plain
left-to-right fold on the CPU.

The claim it rests on: with the running sum |s| = M·u (u = 2^(e-52), M in
[2^52, 2^53)) and a term y of the sign of s written as t·u, fl(s + y) has the
magnitude (M + rnd(t))·u whenever t is not an odd multiple of 1/2 and
M + rnd(t) <= 2^53 - 1.  The restatement follows the device code's steps: 4
terms per lane, 128-term tiles, a scan of the lanes' integer totals, the run
ended by the first tie, sign change, non-finite term or binade overflow, and
ordinary additions from there to the end of the lane (to the end of the tile
after a run shorter than 32 terms).  The GPU side of the same fold is checked
in test_gpu_seq_sums.py."""
import math

import numpy as np
import pytest

from fold_cases import KINDS, grid_ties, terms

PER, TILE = 4, 128
TWO52 = float(2 ** 52)
MAXM = 2 ** 53 - 1


def _bits(x):
    return int(np.float64(x).view(np.uint64))


def _of_bits(b):
    return float(np.uint64(b).view(np.float64))


def seq(xs, acc):
    with np.errstate(over="ignore", invalid="ignore"):
        for v in xs:
            acc = float(np.float64(acc) + np.float64(v))
    return acc


ORDINARY = [0]  # terms the restatement added one after another


def fold_runs(xs, acc):
    xs = np.asarray(xs, np.float64)
    b = len(xs)
    for base in range(0, b, TILE):
        cnt = min(TILE, b - base)
        x = np.zeros(TILE)
        x[:cnt] = xs[base:base + cnt]
        idx = np.arange(TILE)
        q0 = 0
        while q0 < cnt:
            bits = _bits(acc)
            bexp = (bits >> 52) & 0x7FF
            if 64 <= bexp <= 2046:
                neg = acc < 0.0
                scale = _of_bits((2098 - bexp) << 52)
                m = (bits & ((1 << 52) - 1)) | (1 << 52)
                y = -x if neg else x
                with np.errstate(over="ignore", invalid="ignore", under="ignore"):
                    t = y * scale
                    good = (y >= 0.0) & (t < TWO52)
                tg = np.where(good, t, 0.0)
                f = np.floor(tg)
                fr = tg - f
                tie = fr == 0.5
                inside = (idx >= q0) & (idx < cnt)
                c = np.where(inside & good & ~tie,
                             f.astype(np.uint64) + (fr > 0.5).astype(np.uint64), 0)
                pre = np.cumsum(c.astype(object))  # exact integers, in term order
                bad = inside & (~good | tie | (np.array([m + int(p) for p in pre]) > MAXM))
                q = int(np.argmax(bad)) if bad.any() else cnt
                if q > q0:
                    acc = _of_bits((bits & (1 << 63)) | (bexp << 52) | (m + int(pre[q - 1]) - (1 << 52)))
                if q >= cnt:
                    break
                e = cnt if q - q0 < 32 else min(cnt, (q // PER) * PER + PER)
            else:
                q = q0
                e = min(cnt, (q0 // PER) * PER + PER)
            ORDINARY[0] += e - q
            acc = seq(x[q:e], acc)
            q0 = e
    return acc


def _same(a, b):
    return _bits(a) == _bits(b) or (math.isnan(a) and math.isnan(b))


@pytest.mark.parametrize("kind", KINDS)
def test_run_fold_matches_sequential(kind):
    rng = np.random.default_rng(KINDS.index(kind))
    for n in (1, 3, 127, 128, 129, 511, 512, 700, 2000):
        xs = terms(kind, n, rng)
        for acc0 in (0.0, TWO52 - float(rng.integers(0, 1000)),
                     2 * TWO52 - 2.0 * float(rng.integers(0, 1000)), -float(2 ** int(rng.integers(0, 40)))):
            r = seq(xs, acc0)
            f = fold_runs(xs, acc0)
            assert _same(r, f), (kind, n, acc0, r, f)


def test_long_sums_fold_mostly_in_runs():
    # a hub row of 16k weights from zero: the binade changes near the start
    # and at each doubling; all else goes in runs
    xs = np.random.default_rng(1).uniform(0.5, 2.0, 16000)
    ORDINARY[0] = 0
    assert _same(seq(xs, 0.0), fold_runs(xs, 0.0))
    assert ORDINARY[0] < 1000, ORDINARY[0]


def test_run_fold_exact_ties():
    # s = M·2^k and terms (odd)/2 · 2^k: exact ties on s's grid, both signs
    rng = np.random.default_rng(99)
    for _ in range(40):
        acc0, xs = grid_ties(rng, int(rng.integers(1, 400)), int(rng.integers(-20, 20)))
        for a0 in (acc0, -acc0):
            assert _same(seq(xs, a0), fold_runs(xs, a0))


def test_grid_rounding_lemma():
    # fl(s + y) = (M + rnd(t))·u, checked directly on random s and y
    rng = np.random.default_rng(5)
    for _ in range(2000):
        e = int(rng.integers(-30, 30))
        m = (1 << 52) + int(rng.integers(0, 1 << 52))
        s = math.ldexp(float(m), e - 52)
        y = float(rng.random()) * math.ldexp(1.0, e - int(rng.integers(0, 40)))
        t = y * math.ldexp(1.0, 52 - e)
        f = math.floor(t)
        if t - f == 0.5:
            continue
        r = f + (1 if t - f > 0.5 else 0)
        if m + r > MAXM:
            continue
        assert s + y == math.ldexp(float(m + r), e - 52)


def test_oracle_degrees_are_the_sequential_fold():
    # the oracle's k_v is the left-to-right row sum in CSR order
    # (hit_leiden.rs:1063), hub rows included: the value the run fold must
    # reproduce on the GPU
    from fold_cases import seq_fold
    from oracle import oracle as O
    rng = np.random.default_rng(4)
    n = 3000
    src = [rng.integers(0, n, 6000)]
    dst = [rng.integers(0, n, 6000)]
    for hub, deg in ((0, 700), (1, 2500)):
        src.append(np.full(deg, hub))
        dst.append(rng.choice(np.arange(2, n), deg, replace=False))
    s = np.concatenate(src).astype(np.uint32)
    d = np.concatenate(dst).astype(np.uint32)
    g = O.Graph.from_edges(n, s, d, rng.uniform(0.5, 2.0, len(s)))
    off, _, w = g.csr()
    assert np.diff(off).max() >= 2500
    k = g.degrees()
    for v in range(n):
        row = w[off[v]:off[v + 1]]
        want = seq_fold(row, 0.0)
        assert _bits(k[v]) == _bits(want), v
        if len(row) >= 512:
            assert _bits(fold_runs(row, 0.0)) == _bits(want), v
