"""The T-filter's rounding window (refine.cu, k_blocked_bounds): for N positive
FP64 terms the left-to-right sum the reference computes and a sum of the same
terms in any other order differ by less than 8·N·2^-53 times the latter.
Checked here on the CPU for adversarial orders and dynamic ranges."""
import numpy as np
import pytest


def seq_sum(x):
    acc = 0.0
    for v in x:
        acc += float(v)
    return acc


@pytest.mark.parametrize("seed", range(6))
def test_window_covers_order_changes(seed):
    rng = np.random.default_rng(seed)
    for n in [2, 3, 17, 1000, 5000]:
        for dist in ["uniform", "lognormal", "spiky"]:
            if dist == "uniform":
                x = rng.uniform(0.5, 2.0, n)
            elif dist == "lognormal":
                x = rng.lognormal(0.0, 6.0, n)
            else:
                x = np.where(rng.random(n) < 0.01, 1e16, rng.uniform(0.0, 1.0, n)) + 1e-12
            ref = seq_sum(x)
            for order in [np.sort(x), np.sort(x)[::-1], rng.permutation(x)]:
                anyo = seq_sum(order)
                # pairwise (tree) order, as warp reductions produce
                pw = float(np.add.reduce(order))
                for a in (anyo, pw):
                    err = a * n * 2.0 ** -50
                    assert a - err <= ref <= a + err
