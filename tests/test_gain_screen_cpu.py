"""The evaluation kernels screen a vertex's candidates with a division-free
proxy before computing the exact move gain (GainScreen in
hit-leiden_b200/csrc/hl_internal.cuh).  This restates the screen in Python
doubles (every operation rounds to nearest, as the kernels' _rn intrinsics do)
and checks on adversarial near-ties that the screened scan picks the same
winner, with the same gain bits, as the full scan of exact gains
(parallel_frontier.rs:168-200: the largest gain, first position on ties)."""
import math

import numpy as np
import pytest

U16 = 1.7763568394002505e-15  # 16 * 2^-53


def move_gain(w_to, w_cur, tw, gamma, kv, d_cur, d_to):
    a = (w_to - w_cur) / tw
    b = (gamma * kv) * ((d_cur - kv) - d_to)
    return a + b / (tw * tw)


class Screen:
    def __init__(self, w_cur, tw, gamma, kv, d_cur):
        self.tw, self.c, self.g = tw, tw * tw, gamma * kv
        self.dk, self.wcur = d_cur - kv, w_cur
        self.qmax, self.tmax = -math.inf, 0.0

    def keep(self, w_to, d_to):
        p1 = (w_to - self.wcur) * self.c
        p2 = (self.g * (self.dk - d_to)) * self.tw
        q = p1 + p2
        t = abs(p1) + abs(p2)
        margin = U16 * (t + self.tmax) + 1e-300
        if q + margin < self.qmax:
            return False
        if q > self.qmax:
            self.qmax, self.tmax = q, t
        return True


def best(cands, vertex, screened, threads=1):
    """cands: list of (pos, w_to, d_to).  The candidates are dealt to
    `threads` scanners; each keeps (gain, pos); the winners are then merged
    by the same rule, as the kernels' warp and block reductions do."""
    w_cur, tw, gamma, kv, d_cur = vertex
    per = [cands[i::threads] for i in range(threads)]
    out = []
    for part in per:
        sc = Screen(w_cur, tw, gamma, kv, d_cur)
        g, p = -1.0, None
        for pos, w, d in part:
            if screened and not sc.keep(w, d):
                continue
            gn = move_gain(w, w_cur, tw, gamma, kv, d_cur, d)
            if p is None or gn > g or (gn == g and pos < p):
                g, p = gn, pos
        if p is not None:
            out.append((g, p))
    g, p = -1.0, None
    for gn, pos in out:
        if p is None or gn > g or (gn == g and pos < p):
            g, p = gn, pos
    return g, p


def cases(rng, integral):
    for _ in range(400):
        tw = float(rng.integers(10, 10**12)) if integral else rng.uniform(1.0, 1e9)
        kv = float(rng.integers(1, 10**6)) if integral else rng.uniform(0.01, 1e5)
        gamma = float(rng.choice([1.0, 0.5, 2.0, rng.uniform(0.01, 4.0)]))
        d_cur = kv + (float(rng.integers(0, 10**6)) if integral else rng.uniform(0, 1e6))
        w_cur = float(rng.integers(0, 50)) if integral else rng.uniform(0, 50)
        base_w = float(rng.integers(1, 50)) if integral else rng.uniform(0.01, 50)
        base_d = float(rng.integers(1, 10**6)) if integral else rng.uniform(0.01, 1e6)
        cands = []
        for pos in range(int(rng.integers(1, 200))):
            r = rng.random()
            if r < 0.4:  # exact ties of the best-looking candidate
                w, d = base_w, base_d
            elif r < 0.7:  # one ulp (or one unit) away in w or d
                w = np.nextafter(base_w, math.inf if rng.random() < 0.5 else 0.0)
                d = np.nextafter(base_d, math.inf if rng.random() < 0.5 else 0.0)
                if integral:
                    w = base_w + float(rng.integers(-1, 2))
                    d = base_d + float(rng.integers(-1, 2))
                w, d = float(max(w, 0.0)), float(max(d, 0.0))
            else:
                w = float(rng.integers(1, 60)) if integral else rng.uniform(0.01, 60)
                d = float(rng.integers(1, 10**6)) if integral else rng.uniform(0.01, 1e6)
            cands.append((pos, w, d))
        rng.shuffle(cands)
        yield (w_cur, tw, gamma, kv, d_cur), cands


@pytest.mark.parametrize("integral", [True, False])
@pytest.mark.parametrize("threads", [1, 7, 32])
def test_screened_scan_picks_the_exact_winner(integral, threads):
    rng = np.random.default_rng(100 * threads + integral)
    skipped = 0
    for vertex, cands in cases(rng, integral):
        g_full, p_full = best(cands, vertex, False, threads)
        g_scr, p_scr = best(cands, vertex, True, threads)
        assert p_full == p_scr
        assert np.float64(g_full).tobytes() == np.float64(g_scr).tobytes()
        sc = Screen(*vertex)
        skipped += sum(not sc.keep(w, d) for _, w, d in cands)
    assert skipped > 0  # the screen does skip candidates


def test_screen_keeps_every_candidate_within_rounding():
    # candidates whose exact gains collide must all be kept
    vertex = (3.0, 1e6, 1.0, 5.0, 40.0)
    sc = Screen(*vertex)
    kept = [sc.keep(7.0, 11.0) for _ in range(5)]
    assert all(kept)
