"""Seeded synthetic graphs and update batches with the shapes of the benchmark configs.

None of the reference's datasets (SNAP ca-HepTh, uk-2007-05) is available, so
these generators stand in for them with the same sizes and value distributions:

* ``planted``: planted power-law communities with mixing mu, power-law degrees and
  optional triangle closure (config 1: n=9,877, ~21.8k unit edges, mu=0.15,
  clustering ~0.45; config 2 shape: 1M vertices / 20M f64 edges, mu=0.3).
* ``rmat``: R-MAT edge sampling (config 3: scale 25, edge factor 16), produced
  on the GPU with torch as input plumbing.
* batch generators: uniform inserts, degree-preferential inserts and uniform
  deletes of existing edges, all seeded.

Graphs are returned as (n, src, dst, w) numpy arrays with src < dst, no
self-loops and no duplicates.
"""
from __future__ import annotations

import numpy as np


def _powerlaw_int(rng, n, exponent, lo, hi, mean=None):
    """Draw n integers in [lo, hi] from a discrete power law p(x) ~ x^-exponent."""
    xs = np.arange(lo, hi + 1, dtype=np.float64)
    p = xs ** (-exponent)
    p /= p.sum()
    out = rng.choice(xs.astype(np.int64), size=n, p=p)
    if mean is not None and out.mean() > 0:
        scale = mean / out.mean()
        out = np.clip(np.round(out * scale), lo if lo > 0 else 1, hi).astype(np.int64)
    return out


def _community_sizes(rng, n, exponent, lo, hi):
    sizes = []
    total = 0
    while total < n:
        s = int(_powerlaw_int(rng, 1, exponent, lo, hi)[0])
        s = min(s, n - total)
        if s < lo and sizes:
            sizes[-1] += s
        else:
            sizes.append(s)
        total += s
    return np.array(sizes, dtype=np.int64)


def _dedup(n, u, v, w=None):
    a = np.minimum(u, v).astype(np.int64)
    b = np.maximum(u, v).astype(np.int64)
    keep = a != b
    a, b = a[keep], b[keep]
    if w is not None:
        w = w[keep]
    key = a * n + b
    key, idx = np.unique(key, return_index=True)
    a, b = key // n, key % n
    if w is not None:
        w = w[idx]
    return a.astype(np.uint32), b.astype(np.uint32), w


def planted(n, mean_degree, mu, seed, degree_exp=2.5, max_degree=None, comm_exp=1.5,
            comm_min=2, comm_max=400, triangle_frac=0.0, weights=None):
    """Planted-partition graph (LFR-style).

    Each vertex gets a power-law target degree; a fraction 1-mu of its stubs is
    wired inside its community (configuration model), the rest across the whole
    graph.  ``triangle_frac`` of the intra edges are instead placed by closing
    wedges, which raises the clustering coefficient.  ``weights`` = None gives
    unit weights, or a (lo, hi) pair for uniform f64 weights.
    """
    rng = np.random.default_rng(seed)
    if max_degree is None:
        max_degree = max(8, int(np.sqrt(n) * 4))
    deg = _powerlaw_int(rng, n, degree_exp, 1, max_degree, mean=mean_degree)
    sizes = _community_sizes(rng, n, comm_exp, comm_min, comm_max)
    perm = rng.permutation(n)
    comm = np.empty(n, np.int64)
    starts = np.concatenate([[0], np.cumsum(sizes)])
    for c in range(len(sizes)):
        comm[perm[starts[c]:starts[c + 1]]] = c
    intra = rng.binomial(deg, 1.0 - mu)
    inter = deg - intra
    # Intra edges: shuffle stubs inside each community and pair them up.
    order = np.argsort(comm, kind="stable")
    stub_node = np.repeat(order, intra[order])
    stub_comm = comm[stub_node]
    key = stub_comm * 4.0 + rng.random(len(stub_node))
    stub_node = stub_node[np.argsort(key, kind="stable")]
    stub_comm = comm[stub_node]
    m_pairs = len(stub_node) // 2
    a, b = stub_node[0:2 * m_pairs:2], stub_node[1:2 * m_pairs:2]
    same = comm[a] == comm[b]
    iu, iv = a[same], b[same]
    n_tri = int(len(iu) * triangle_frac)
    if n_tri > 0:
        iu, iv = iu[n_tri:], iv[n_tri:]
    # Inter edges: global configuration model.
    sn = np.repeat(np.arange(n), inter)
    rng.shuffle(sn)
    mp = len(sn) // 2
    ou, ov = sn[0:2 * mp:2], sn[1:2 * mp:2]
    u = np.concatenate([iu, ou])
    v = np.concatenate([iv, ov])
    if n_tri > 0:
        # Close wedges: pick a vertex, two of its current intra neighbours.
        a0, b0, _ = _dedup(n, u, v)
        nb_src = np.concatenate([a0, b0]).astype(np.int64)
        nb_dst = np.concatenate([b0, a0]).astype(np.int64)
        same = comm[nb_src] == comm[nb_dst]
        nb_src, nb_dst = nb_src[same], nb_dst[same]
        o = np.argsort(nb_src, kind="stable")
        nb_src, nb_dst = nb_src[o], nb_dst[o]
        cnt = np.bincount(nb_src, minlength=n)
        off = np.concatenate([[0], np.cumsum(cnt)])
        cand = np.nonzero(cnt >= 2)[0]
        centers = cand[rng.integers(0, len(cand), size=n_tri)]
        c0 = off[centers]
        dc = cnt[centers]
        x = rng.integers(0, dc)
        y = (x + 1 + rng.integers(0, np.maximum(dc - 1, 1))) % dc
        tu, tv = nb_dst[c0 + x], nb_dst[c0 + y]
        u = np.concatenate([u, tu])
        v = np.concatenate([v, tv])
    w = None
    if weights is not None:
        w = rng.uniform(weights[0], weights[1], size=len(u))
    src, dst, w = _dedup(n, u, v, w)
    if w is None:
        w = np.ones(len(src), np.float64)
    return n, src, dst, w.astype(np.float64), comm.astype(np.uint32)


def config1(seed=0):
    """n=9,877, ~21.8k unit edges, ~480 communities (sizes 2-400, exp 1.5),
    mu=0.15, power-law degrees (exp 2.5, mean 4.4), triangle closure."""
    n, s, d, w, comm = planted(9877, 5.3, 0.15, seed, degree_exp=2.5, max_degree=65,
                               comm_exp=1.5, comm_min=2, comm_max=400, triangle_frac=0.35)
    return n, s, d, w


def config2(seed=0, n=1_000_000, mean_degree=40.0):
    """LFR-style 1M vertices / ~20M edges, degree exp 2.5 (mean 40, max 2000),
    community sizes exp 1.5 in [50, 5000], mu=0.3, f64 weights U[0.5, 2.0]."""
    n, s, d, w, comm = planted(n, mean_degree * 1.13, 0.3, seed, degree_exp=2.5, max_degree=2000,
                               comm_exp=1.5, comm_min=50, comm_max=5000, weights=(0.5, 2.0))
    return n, s, d, w


def uniform_inserts(n, k, seed, existing=None):
    """k uniformly random new undirected unit edges (no self-loops)."""
    rng = np.random.default_rng(seed)
    out_u, out_v = [], []
    seen = set()
    ex = existing
    while len(out_u) < k:
        a = rng.integers(0, n, size=2 * k)
        b = rng.integers(0, n, size=2 * k)
        for x, y in zip(a.tolist(), b.tolist()):
            if x == y:
                continue
            key = (min(x, y), max(x, y))
            if key in seen or (ex is not None and key in ex):
                continue
            seen.add(key)
            out_u.append(key[0])
            out_v.append(key[1])
            if len(out_u) == k:
                break
    return (np.array(out_u, np.uint32), np.array(out_v, np.uint32), np.ones(k, np.float64))


class EdgeStore:
    """Current weighted edge set of a dynamic graph (for generating deletes)."""

    def __init__(self, n, src, dst, w):
        self.n = n
        self.key = (src.astype(np.int64) * n + dst.astype(np.int64))
        self.w = w.astype(np.float64).copy()
        self.deg = np.bincount(src, minlength=n) + np.bincount(dst, minlength=n)
        self.extra = {}
        self.removed = set()

    def weight(self, a, b):
        key = a * self.n + b
        if key in self.extra:
            return self.extra[key]
        if key in self.removed:
            return None
        i = np.searchsorted(self.key, key)
        if i < len(self.key) and self.key[i] == key:
            return float(self.w[i])
        return None

    def apply(self, u, v, w):
        for a, b, x in zip(u.tolist(), v.tolist(), w.tolist()):
            a, b = min(a, b), max(a, b)
            cur = self.weight(a, b)
            new = (cur or 0.0) + x
            key = a * self.n + b
            if new > 1e-12:
                self.extra[key] = new
                self.removed.discard(key)
            else:
                self.extra.pop(key, None)
                self.removed.add(key)

    def random_existing(self, rng, k):
        """k distinct edges of the base edge set that are still present, drawn
        uniformly, with their current weights."""
        out = []
        chosen = set()
        while len(out) < k:
            idx = rng.integers(0, len(self.key), size=2 * (k - len(out)) + 8)
            for i in idx.tolist():
                key = int(self.key[i])
                if key in chosen or key in self.removed:
                    continue
                w = self.extra.get(key, float(self.w[i]))
                a, b = divmod(key, self.n)
                out.append((a, b, w))
                chosen.add(key)
                if len(out) == k:
                    break
        return out


def mixed_batch(store: EdgeStore, k, insert_frac, seed, weights=None, preferential=True):
    """k updates: insert_frac new edges (endpoints drawn by degree when
    ``preferential``, uniform otherwise) and the rest deletes of existing edges
    chosen uniformly (alpha = -current weight, which removes the edge)."""
    rng = np.random.default_rng(seed)
    n = store.n
    ki = int(round(k * insert_frac))
    kd = k - ki
    if preferential:
        p = store.deg.astype(np.float64) + 1.0
        p /= p.sum()
        a = rng.choice(n, size=2 * ki + 64, p=p)
        b = rng.choice(n, size=2 * ki + 64, p=p)
    else:
        a = rng.integers(0, n, size=2 * ki + 64)
        b = rng.integers(0, n, size=2 * ki + 64)
    iu, iv = [], []
    seen = set()
    for x, y in zip(a.tolist(), b.tolist()):
        if len(iu) == ki:
            break
        if x == y:
            continue
        key = (min(x, y), max(x, y))
        if key in seen:
            continue
        seen.add(key)
        iu.append(key[0])
        iv.append(key[1])
    if weights is None:
        iw = np.ones(len(iu))
    else:
        iw = rng.uniform(weights[0], weights[1], size=len(iu))
    dels = store.random_existing(rng, kd)
    u = np.array(iu + [x[0] for x in dels], np.uint32)
    v = np.array(iv + [x[1] for x in dels], np.uint32)
    w = np.concatenate([iw, np.array([-x[2] for x in dels])]).astype(np.float64)
    perm = rng.permutation(len(u))
    u, v, w = u[perm], v[perm], w[perm]
    store.apply(u, v, w)
    return u, v, w


def rmat_torch(scale, edge_factor, seed, a=0.57, b=0.19, c=0.19, device="cuda"):
    """R-MAT edge list generated on the GPU with torch (input plumbing only):
    symmetrised (src < dst), duplicates and self-loops removed.  Returns
    device tensors (src, dst) of dtype int32 sorted by (src, dst)."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    n = 1 << scale
    m = n * edge_factor
    chunk = 1 << 26
    keys = []
    for start in range(0, m, chunk):
        cnt = min(chunk, m - start)
        src = torch.zeros(cnt, dtype=torch.int64, device=device)
        dst = torch.zeros(cnt, dtype=torch.int64, device=device)
        for lvl in range(scale):
            r = torch.rand(cnt, generator=g, device=device)
            bit_s = (r >= a + b).to(torch.int64)
            bit_d = (((r >= a) & (r < a + b)) | (r >= a + b + c)).to(torch.int64)
            src |= bit_s << lvl
            dst |= bit_d << lvl
        lo = torch.minimum(src, dst)
        hi = torch.maximum(src, dst)
        keep = lo != hi
        keys.append(lo[keep] * n + hi[keep])
        del src, dst, lo, hi
    key = torch.unique(torch.cat(keys))
    return n, (key // n).to(torch.int32), (key % n).to(torch.int32)


def rmat_batch_torch(scale, base_src, base_dst, k, insert_frac, seed, a=0.57, b=0.19, c=0.19):
    """k unit updates on the GPU: insert_frac R-MAT-sampled pairs (self-loops
    redrawn as the pair's next sample is not needed: they are dropped and the
    batch is topped up with uniform pairs) and the rest deletes of base edges
    drawn uniformly (weight -1; deleting an edge that is already gone is a
    no-op).  Returns int32 device tensors (src, dst) and an f64 tensor w."""
    import torch
    dev = base_src.device
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    n = 1 << scale
    ki = int(round(k * insert_frac))
    kd = k - ki
    src = torch.zeros(ki, dtype=torch.int64, device=dev)
    dst = torch.zeros(ki, dtype=torch.int64, device=dev)
    for lvl in range(scale):
        r = torch.rand(ki, generator=g, device=dev)
        src |= (r >= a + b).to(torch.int64) << lvl
        dst |= (((r >= a) & (r < a + b)) | (r >= a + b + c)).to(torch.int64) << lvl
    loop = src == dst
    if bool(loop.any()):
        fix = torch.randint(0, n - 1, (int(loop.sum()),), generator=g, device=dev)
        dst[loop] = fix + (fix >= src[loop]).to(torch.int64)
    di = torch.randint(0, base_src.numel(), (kd,), generator=g, device=dev)
    u = torch.cat([torch.minimum(src, dst).to(torch.int32), base_src[di]])
    v = torch.cat([torch.maximum(src, dst).to(torch.int32), base_dst[di]])
    w = torch.cat([torch.ones(ki, dtype=torch.float64, device=dev),
                   -torch.ones(kd, dtype=torch.float64, device=dev)])
    return u.contiguous(), v.contiguous(), w.contiguous()


def _loguniform_int(rng, lo, hi, size):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size)).astype(np.int64)


def config4(seed=0, count=256):
    """Batching form: `count` independent graphs, vertex counts log-uniform in
    [1k, 200k], planted power-law communities with mu log-uniform in
    [0.1, 0.4], target mean degree uniform in [4, 32], unit weights."""
    rng = np.random.default_rng(seed)
    ns = _loguniform_int(rng, 1000, 200_000, count)
    mus = np.exp(rng.uniform(np.log(0.1), np.log(0.4), count))
    degs = rng.uniform(4.0, 32.0, count)
    out = []
    for i in range(count):
        n, s, d, w, _ = planted(int(ns[i]), float(degs[i]), float(mus[i]), seed * 100_000 + i,
                                comm_min=5, comm_max=400)
        out.append((n, s, d, w))
    return out


def fast_batch(n, src, dst, k, insert_frac, seed):
    """k unit updates: insert_frac uniform random new pairs (u != v; a pair
    that already exists is strengthened) and the rest deletes of base edges
    drawn uniformly (weight -1; deleting an edge an earlier batch already
    removed is a no-op).  Vectorised, for large request streams."""
    rng = np.random.default_rng(seed)
    ki = int(round(k * insert_frac))
    kd = k - ki
    a = rng.integers(0, n, size=ki, dtype=np.int64)
    b = rng.integers(0, n - 1, size=ki, dtype=np.int64)
    b = b + (b >= a)  # b != a
    di = rng.integers(0, len(src), size=kd) if len(src) else np.zeros(0, np.int64)
    u = np.concatenate([np.minimum(a, b), src[di].astype(np.int64)]).astype(np.uint32)
    v = np.concatenate([np.maximum(a, b), dst[di].astype(np.int64)]).astype(np.uint32)
    w = np.concatenate([np.ones(ki), -np.ones(kd)])
    return u, v, w


def config5(seed=0, count=32, scale=1.0):
    """Serving form: `count` resident graphs, vertex counts log-uniform in
    [100k, 5M] (times `scale`), planted communities, mu 0.25, target mean
    degree 16, unit weights."""
    rng = np.random.default_rng(seed)
    ns = _loguniform_int(rng, max(1000, int(100_000 * scale)), max(2000, int(5_000_000 * scale)),
                         count)
    out = []
    for i in range(count):
        n, s, d, w, _ = planted(int(ns[i]), 16.0, 0.25, seed * 100_000 + 50_000 + i,
                                comm_min=5, comm_max=2000)
        out.append((n, s, d, w))
    return out
