"""Term generators for the ordered f64 sum tests (CPU restatement and GPU)."""
import numpy as np

KINDS = ["weights", "degrees", "dyadic", "mixed", "negative", "wide", "zeros", "tiny", "huge",
         "nonfinite"]


def terms(kind, n, rng):
    """n terms of one family: graph weights, degrees, dyadic values with zeros,
    mixed signs, negatives, a wide exponent range, signed zeros, subnormals,
    values that overflow, and a sprinkling of NaN and infinity."""
    u = rng.random(n)
    if kind == "weights":
        return 0.5 + 1.5 * u
    if kind == "degrees":
        return 1.0 + 1e6 * u
    if kind == "dyadic":
        return rng.integers(0, 8, n) * 0.25
    if kind == "mixed":
        return (u - 0.5) * 4
    if kind == "negative":
        return -(0.5 + 1.5 * u)
    if kind == "wide":
        return np.ldexp(1.0 + u, rng.integers(-60, 60, n))
    if kind == "zeros":
        return np.where(rng.random(n) < 0.3, -0.0, np.where(rng.random(n) < 0.2, 0.0, 1.0 + u))
    if kind == "tiny":
        return np.ldexp(1.0 + u, rng.integers(-1074, -1010, n))
    if kind == "huge":
        return np.ldexp(1.0 + u, rng.integers(1000, 1023, n))
    if kind == "nonfinite":
        return np.where(rng.random(n) < 0.01, np.where(rng.random(n) < 0.5, np.nan, np.inf), 0.5 + u)
    raise ValueError(kind)


def grid_ties(rng, n, k):
    """A start s = M·2^k (M in [2^52, 2^53)) and n terms on s's grid, a quarter
    of them exact ties (odd multiples of 2^(k-1))."""
    m = (1 << 52) + int(rng.integers(0, 1 << 51))
    odd = 2 * rng.integers(0, 50, n) + 1
    xs = np.where(rng.random(n) < 0.25, np.ldexp(odd.astype(float), k - 1),
                  np.ldexp(rng.integers(0, 100, n).astype(float), k - 2))
    return float(np.ldexp(float(m), k)), xs


def seq_fold(xs, acc):
    """acc + xs[0] + xs[1] + ... left to right (numpy's accumulate is a
    sequential loop)."""
    with np.errstate(over="ignore", invalid="ignore"):
        return float(np.add.accumulate(np.concatenate([[acc], np.asarray(xs, np.float64)]))[-1])
