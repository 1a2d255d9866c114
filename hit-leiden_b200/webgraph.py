"""WebGraph (BV) graphs in the reference's loader conventions.

The reference's benchmark reads its datasets (uk-2007-05@100000, SNAP graphs
converted to BV) with the `webgraph` crate 0.6.0 (``Cargo.toml:32``):
``BvGraphSeq::with_basename(path).load()``, then keeps every arc ``src < dst``
as an unweighted undirected edge and skips self-loops
(``src/main.rs:189-230``).  That crate is not vendored, so this module
restates the BV format it reads, from the published description (Boldi and
Vigna, "The WebGraph Framework I: Compression Techniques", WWW 2004, and the
format's reference implementation conventions):

* ``<basename>.properties``: ``nodes``, ``arcs``, ``windowsize``,
  ``maxrefcount``, ``minintervallength``, ``zetak``, ``compressionflags``;
* ``<basename>.graph``: one bit stream, most significant bit first.  Per node
  x: its outdegree; if nonzero, a reference r (0 = none) to the list of node
  x - r, then the copy blocks over that list (alternately copied and skipped,
  the first block's length as is, later ones minus one, the rest copied when
  the block count is even); the intervals (count, then the first left
  extreme as a signed gap from x and later ones as gaps after the previous
  interval, lengths minus minintervallength); the residuals (the first as a
  signed gap from x, later ones as gaps minus one).  Default codes: gamma
  for outdegrees, blocks, block counts and intervals; unary for references;
  zeta_k for residuals (``compressionflags`` may name others).

``write_bvgraph`` is the matching encoder (greedy reference choice in the
window), used by the tests and to convert edge lists.  Plain Python: a
loader, not part of the update path.
"""
from __future__ import annotations

import os
from typing import Dict, List, Optional, Sequence

import numpy as np

_DEFAULT_CODES = {"OUTDEGREES": "GAMMA", "REFERENCES": "UNARY", "BLOCKS": "GAMMA",
                  "BLOCK_COUNT": "GAMMA", "RESIDUALS": "ZETA", "OFFSETS": "GAMMA"}


def _nat2int(x: int) -> int:
    return x >> 1 if (x & 1) == 0 else -((x + 1) >> 1)


def _int2nat(x: int) -> int:
    return 2 * x if x >= 0 else -2 * x - 1


class _BitReader:
    """Most-significant-bit-first reader over a bytes object."""

    def __init__(self, data: bytes):
        self.data = data
        self.pos = 0  # bit position

    def bit(self) -> int:
        p = self.pos
        if (p >> 3) >= len(self.data):
            raise ValueError("BV stream ends early")
        self.pos = p + 1
        return (self.data[p >> 3] >> (7 - (p & 7))) & 1

    def bits(self, n: int) -> int:
        x = 0
        for _ in range(n):
            x = (x << 1) | self.bit()
        return x

    def unary(self) -> int:
        n = 0
        while self.bit() == 0:
            n += 1
        return n

    def gamma(self) -> int:
        msb = self.unary()
        return ((1 << msb) | self.bits(msb)) - 1

    def delta(self) -> int:
        msb = self.gamma()
        return ((1 << msb) | self.bits(msb)) - 1

    def zeta(self, k: int) -> int:
        h = self.unary()
        left = 1 << (h * k)
        m = self.bits(h * k + k - 1)
        if m < left:
            return m + left - 1
        return (m << 1) + self.bit() - 1

    def code(self, name: str, k: int) -> int:
        if name == "GAMMA":
            return self.gamma()
        if name == "DELTA":
            return self.delta()
        if name == "UNARY":
            return self.unary()
        if name == "ZETA":
            return self.zeta(k)
        raise ValueError(f"unsupported BV code {name}")


class _BitWriter:
    def __init__(self):
        self.out = bytearray()
        self.cur = 0
        self.n = 0  # bits in cur

    def bit(self, b: int) -> None:
        self.cur = (self.cur << 1) | (b & 1)
        self.n += 1
        if self.n == 8:
            self.out.append(self.cur)
            self.cur = 0
            self.n = 0

    def bits(self, x: int, n: int) -> None:
        for i in range(n - 1, -1, -1):
            self.bit((x >> i) & 1)

    def unary(self, x: int) -> None:
        for _ in range(x):
            self.bit(0)
        self.bit(1)

    def gamma(self, x: int) -> None:
        x += 1
        msb = x.bit_length() - 1
        self.unary(msb)
        self.bits(x, msb)

    def delta(self, x: int) -> None:
        x += 1
        msb = x.bit_length() - 1
        self.gamma(msb)
        self.bits(x, msb)

    def zeta(self, x: int, k: int) -> None:
        x += 1
        msb = x.bit_length() - 1
        h = msb // k
        self.unary(h)
        left = 1 << (h * k)
        if x - left < left:
            self.bits(x - left, h * k + k - 1)
        else:
            self.bits(x, h * k + k)

    def code(self, name: str, x: int, k: int) -> None:
        if name == "GAMMA":
            self.gamma(x)
        elif name == "DELTA":
            self.delta(x)
        elif name == "UNARY":
            self.unary(x)
        elif name == "ZETA":
            self.zeta(x, k)
        else:
            raise ValueError(f"unsupported BV code {name}")

    def getvalue(self) -> bytes:
        if self.n:
            return bytes(self.out) + bytes([self.cur << (8 - self.n)])
        return bytes(self.out)


def read_properties(path: str) -> Dict[str, str]:
    """A Java-style properties file: ``key=value`` (or ``key: value``)."""
    props = {}
    for raw in open(path, encoding="utf-8"):
        line = raw.strip()
        if not line or line[0] in "#!":
            continue
        for sep in ("=", ":"):
            if sep in line:
                k, v = line.split(sep, 1)
                props[k.strip()] = v.strip()
                break
    return props


def _codes(flags: str) -> Dict[str, str]:
    codes = dict(_DEFAULT_CODES)
    for part in flags.replace(" ", "").split("|"):
        if not part:
            continue
        comp, _, code = part.rpartition("_")
        if comp not in codes:
            raise ValueError(f"unknown compression flag {part}")
        codes[comp] = code
    return codes


def read_bvgraph(basename: str) -> List[np.ndarray]:
    """Successor lists of every node of ``<basename>.graph`` (ascending)."""
    props = read_properties(basename + ".properties")
    n = int(props["nodes"])
    window = int(props.get("windowsize", 7))
    min_interval = int(props.get("minintervallength", 4))
    k = int(props.get("zetak", 3))
    codes = _codes(props.get("compressionflags", ""))
    rd = _BitReader(open(basename + ".graph", "rb").read())
    succ: List[np.ndarray] = []
    for x in range(n):
        d = rd.code(codes["OUTDEGREES"], k)
        if d == 0:
            succ.append(np.zeros(0, np.int64))
            continue
        ref = rd.code(codes["REFERENCES"], k) if window > 0 else 0
        copied: List[int] = []
        extra = d
        if ref > 0:
            if ref > x:
                raise ValueError(f"node {x}: reference {ref} before the first node")
            rlist = succ[x - ref]
            nblocks = rd.code(codes["BLOCK_COUNT"], k)
            blocks = [rd.code(codes["BLOCKS"], k) + (1 if i else 0) for i in range(nblocks)]
            p = 0
            for i, b in enumerate(blocks):
                if i % 2 == 0:
                    copied.extend(rlist[p:p + b].tolist())
                p += b
            if nblocks % 2 == 0:
                copied.extend(rlist[p:].tolist())
            extra = d - len(copied)
        vals: List[int] = []
        if extra > 0 and min_interval > 0:
            nint = rd.gamma()
            prev = 0
            for i in range(nint):
                if i == 0:
                    left = _nat2int(rd.gamma()) + x
                else:
                    left = rd.gamma() + prev + 1  # a gap of at least one id
                ln = rd.gamma() + min_interval
                vals.extend(range(left, left + ln))
                prev = left + ln  # one past the interval
                extra -= ln
        if extra < 0:
            raise ValueError(f"node {x}: inconsistent outdegree")
        prev = 0
        for i in range(extra):
            if i == 0:
                prev = _nat2int(rd.code(codes["RESIDUALS"], k)) + x
            else:
                prev = rd.code(codes["RESIDUALS"], k) + prev + 1
            vals.append(prev)
        lst = np.array(sorted(copied + vals), np.int64)
        if len(lst) != d or (len(lst) and (lst[0] < 0 or lst[-1] >= n)):
            raise ValueError(f"node {x}: corrupt successor list")
        succ.append(lst)
    return succ


def _intervals(extra: Sequence[int], min_len: int):
    """Maximal runs of consecutive ids of length >= min_len, and the rest."""
    runs, rest = [], []
    i = 0
    while i < len(extra):
        j = i
        while j + 1 < len(extra) and extra[j + 1] == extra[j] + 1:
            j += 1
        if min_len > 0 and j - i + 1 >= min_len:
            runs.append((extra[i], j - i + 1))
        else:
            rest.extend(extra[i:j + 1])
        i = j + 1
    return runs, rest


def _encode_node(w: _BitWriter, x: int, lst: List[int], rlist: Optional[List[int]], ref: int,
                 codes, k: int, window: int, min_interval: int) -> None:
    w.code(codes["OUTDEGREES"], len(lst), k)
    if not lst:
        return
    extra = lst
    if window > 0:
        w.code(codes["REFERENCES"], ref, k)
    if ref > 0:
        inlist = set(lst)
        flags = [v in inlist for v in rlist]
        blocks = []
        cur, run = True, 0
        for fl in flags:
            if fl == cur:
                run += 1
            else:
                blocks.append(run)
                cur, run = fl, 1
        blocks.append(run)
        # the last block is implicit: the reader copies the rest of the list
        # when the count of explicit blocks is even, and skips it otherwise
        blocks.pop()
        w.code(codes["BLOCK_COUNT"], len(blocks), k)
        for i, b in enumerate(blocks):
            w.code(codes["BLOCKS"], b - (1 if i else 0), k)
        cset = {v for v, fl in zip(rlist, flags) if fl}
        extra = [v for v in lst if v not in cset]
    if extra and min_interval > 0:
        runs, rest = _intervals(extra, min_interval)
        w.gamma(len(runs))
        prev = 0
        for i, (left, ln) in enumerate(runs):
            if i == 0:
                w.gamma(_int2nat(left - x))
            else:
                w.gamma(left - prev - 1)
            w.gamma(ln - min_interval)
            prev = left + ln
        extra = rest
    prev = 0
    for i, v in enumerate(extra):
        if i == 0:
            w.code(codes["RESIDUALS"], _int2nat(v - x), k)
        else:
            w.code(codes["RESIDUALS"], v - prev - 1, k)
        prev = v


def write_bvgraph(basename: str, succ: Sequence[Sequence[int]], window: int = 7,
                  max_ref_count: int = 3, min_interval: int = 4, zeta_k: int = 3,
                  flags: str = "") -> dict:
    """Write successor lists (each ascending, no duplicates) as a BV graph,
    with the default codes unless ``flags`` names others (for example
    ``"RESIDUALS_GAMMA|OUTDEGREES_DELTA"``).  Each node references the
    window's list that encodes it in the fewest bits (reference chains at most
    ``max_ref_count`` long).  Returns counts of the features used."""
    codes = _codes(flags)
    lists = [sorted(int(v) for v in s) for s in succ]
    n = len(lists)
    out = _BitWriter()
    chain = [0] * n
    used = {"references": 0, "intervals": 0, "arcs": 0}
    for x, lst in enumerate(lists):
        best_ref, best_bits = 0, None
        for r in range(0, min(window, x) + 1 if window > 0 else 1):
            if r > 0 and (chain[x - r] >= max_ref_count or not lists[x - r]):
                continue
            trial = _BitWriter()
            _encode_node(trial, x, lst, lists[x - r] if r else None, r, codes, zeta_k, window,
                         min_interval)
            nb = len(trial.out) * 8 + trial.n
            if best_bits is None or nb < best_bits:
                best_ref, best_bits = r, nb
        if not lst:
            best_ref = 0
        chain[x] = chain[x - best_ref] + 1 if best_ref else 0
        _encode_node(out, x, lst, lists[x - best_ref] if best_ref else None, best_ref, codes,
                     zeta_k, window, min_interval)
        used["references"] += best_ref > 0
        if lst and min_interval > 0:
            extra = lst
            if best_ref:
                rs = set(lists[x - best_ref])
                extra = [v for v in lst if v not in rs]
            used["intervals"] += len(_intervals(extra, min_interval)[0])
        used["arcs"] += len(lst)
    with open(basename + ".graph", "wb") as fh:
        fh.write(out.getvalue())
    with open(basename + ".properties", "w", encoding="utf-8") as fh:
        fh.write(f"nodes={n}\narcs={used['arcs']}\nwindowsize={window}\n"
                 f"maxrefcount={max_ref_count}\nminintervallength={min_interval}\n"
                 f"zetak={zeta_k}\ncompressionflags={flags}\nversion=0\n"
                 "graphclass=it.unimi.dsi.webgraph.BVGraph\n")
    return used


def load_webgraph(basename: str):
    """The reference's ``load_webgraph`` (src/main.rs:189-230): every arc with
    ``src < dst`` becomes one unweighted undirected edge; self-loops are
    skipped (and counted); ``node_count`` is the graph's node count."""
    from .io import EdgeList
    succ = read_bvgraph(basename)
    n = len(succ)
    src, dst = [], []
    loops = 0
    for x, lst in enumerate(succ):
        loops += int(np.count_nonzero(lst == x))
        keep = lst[lst > x]
        src.append(np.full(len(keep), x, np.uint32))
        dst.append(keep.astype(np.uint32))
    s = np.concatenate(src) if src else np.zeros(0, np.uint32)
    d = np.concatenate(dst) if dst else np.zeros(0, np.uint32)
    return EdgeList(os.path.basename(basename), n, s, d, np.ones(len(s)), loops)
