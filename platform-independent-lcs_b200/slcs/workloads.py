"""Seeded synthetic workloads for the five benchmark configurations.

The reference publishes no dataset for this path; its own driver draws binary
strings from std::mt19937 (src/test_utility.hpp:8-18).  The configurations
below follow the shapes, sizes and value distributions of the benchmark
definitions, generated from numpy's PCG64 so that every machine with the same
numpy produces byte-identical inputs.

  pair_4096           4096 x 4096, i.i.d. uniform over {0..3}
  pair_131072_mutated 131072 x 131072, b = mutate(a) (10% subs, 1%+1% indels)
  pair_1M             1048576 x 1048576, i.i.d. uniform over {0..3}
  reads_20000         20,000 read-vs-window pairs, lognormal read lengths
  sweep shapes        log-uniform m, n in [64, 262144], alphabets {2,4,20,256}
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def uniform(rng: np.random.Generator, length: int, sigma: int = 4) -> np.ndarray:
    return rng.integers(0, sigma, size=length, dtype=np.uint8)


def mutate(rng: np.random.Generator, s: np.ndarray, sub: float, ins: float, dele: float,
           sigma: int = 4, mean_indel: float = 3.0) -> np.ndarray:
    """Copy of s with substitutions (a uniformly drawn different symbol) and
    insertions/deletions whose lengths are geometric with the given mean."""
    n = len(s)
    out = s.copy()
    if sub > 0 and sigma > 1:
        pos = np.nonzero(rng.random(n) < sub)[0]
        shift = rng.integers(1, sigma, size=len(pos), dtype=np.int64)
        out[pos] = ((out[pos].astype(np.int64) + shift) % sigma).astype(np.uint8)
    ev = rng.random(n)
    ins_pos = np.nonzero(ev < ins)[0]
    del_pos = np.nonzero((ev >= ins) & (ev < ins + dele))[0]
    p = 1.0 / mean_indel
    pieces = []
    cur = 0
    events = sorted([(int(i), 0) for i in ins_pos] + [(int(i), 1) for i in del_pos])
    for pos, kind in events:
        if pos < cur:
            continue
        pieces.append(out[cur:pos])
        length = int(rng.geometric(p))
        if kind == 0:
            pieces.append(uniform(rng, length, sigma))
            cur = pos
        else:
            cur = min(n, pos + length)
    pieces.append(out[cur:])
    return np.concatenate(pieces) if pieces else out


def fit_length(rng: np.random.Generator, s: np.ndarray, length: int, sigma: int = 4) -> np.ndarray:
    if len(s) >= length:
        return s[:length].copy()
    return np.concatenate([s, uniform(rng, length - len(s), sigma)])


def pair_4096(seed: int = 1):
    rng = np.random.default_rng(seed)
    return uniform(rng, 4096), uniform(rng, 4096)


def pair_131072_mutated(seed: int = 2):
    rng = np.random.default_rng(seed)
    a = uniform(rng, 131072)
    b = fit_length(rng, mutate(rng, a, 0.10, 0.01, 0.01), 131072)
    return a, b


def pair_1m(seed: int = 3):
    rng = np.random.default_rng(seed)
    return uniform(rng, 1 << 20), uniform(rng, 1 << 20)


@dataclass
class Batch:
    """A packed batch: pair p is a_blob[a_off[p]:+ms[p]] against b_blob[b_off[p]:+ns[p]].
    Offsets are multiples of 16 so that vector loads of any pair stay aligned."""
    a_blob: np.ndarray
    b_blob: np.ndarray
    a_off: np.ndarray
    b_off: np.ndarray
    ms: np.ndarray
    ns: np.ndarray

    @property
    def npairs(self) -> int:
        return len(self.ms)

    @property
    def cells(self) -> int:
        return int(np.sum(self.ms.astype(np.int64) * self.ns.astype(np.int64)))

    def strand_offsets(self):
        """Offsets of each pair's (h, v) strands in a packed output blob."""
        sizes = self.ms.astype(np.int64) + self.ns.astype(np.int64)
        off = np.zeros(len(sizes), np.int64)
        if len(sizes) > 1:
            off[1:] = np.cumsum(sizes)[:-1]
        return off, int(sizes.sum())

    def pair(self, p: int):
        a = self.a_blob[self.a_off[p]:self.a_off[p] + self.ms[p]]
        b = self.b_blob[self.b_off[p]:self.b_off[p] + self.ns[p]]
        return a, b

    def subset(self, indices) -> "Batch":
        """The pairs at `indices` (in that order), packed into a batch of their own."""
        return pack([self.pair(int(p)) for p in indices])


def pack(pairs) -> Batch:
    """Pack a list of (a, b) uint8 arrays with 16-byte aligned offsets."""
    ms = np.array([len(a) for a, _ in pairs], np.int32)
    ns = np.array([len(b) for _, b in pairs], np.int32)

    def blob(strings):
        lens = np.array([len(s) for s in strings], np.int64)
        padded = (lens + 15) // 16 * 16
        off = np.zeros(len(strings), np.int64)
        if len(strings) > 1:
            off[1:] = np.cumsum(padded)[:-1]
        total = int(padded.sum()) + 16
        buf = np.zeros(total, np.uint8)
        for o, s in zip(off, strings):
            buf[o:o + len(s)] = s
        return buf, off

    a_blob, a_off = blob([a for a, _ in pairs])
    b_blob, b_off = blob([b for _, b in pairs])
    return Batch(a_blob, b_blob, a_off, b_off, ms, ns)


def reads_20000(seed: int = 4, npairs: int = 20000) -> Batch:
    """Read-versus-window pairs: read length ~ lognormal(mean 150, sd 60) clipped
    to [50, 1000]; window = read_len * U(1.0, 1.5) uniform symbols over {0..3};
    the read is a substring of the window with 5% substitutions and 1% indels.
    a = read, b = window."""
    rng = np.random.default_rng(seed)
    mean, sd = 150.0, 60.0
    sigma_ln = math.sqrt(math.log(1.0 + sd * sd / (mean * mean)))
    mu_ln = math.log(mean * mean / math.sqrt(mean * mean + sd * sd))
    read_len = np.clip(np.round(rng.lognormal(mu_ln, sigma_ln, npairs)), 50, 1000).astype(np.int64)
    win_len = np.round(read_len * rng.uniform(1.0, 1.5, npairs)).astype(np.int64)
    pairs = []
    for p in range(npairs):
        w = uniform(rng, int(win_len[p]))
        start = int(rng.integers(0, win_len[p] - read_len[p] + 1))
        read = w[start:start + read_len[p]]
        read = mutate(rng, read, 0.05, 0.005, 0.005)
        if len(read) == 0:
            read = uniform(rng, 1)
        pairs.append((read, w))
    return pack(pairs)


@dataclass
class Shape:
    m: int
    n: int
    sigma: int
    mutated: bool
    batch: int
    seed: int

    @property
    def cells(self) -> int:
        return self.m * self.n * self.batch


def sweep_shapes(count: int, seed: int, cell_cap: float = 2.0e9):
    """Shapes of the cost-model sweep: m, n log-uniform in [64, 262144], alphabet
    from {2, 4, 20, 256}, i.i.d. or mutated content, batch log-uniform in
    [1, 4096].  The batch is scaled down until m*n*batch <= cell_cap (the stated
    per-shape cell budget), keeping at least one pair."""
    rng = np.random.default_rng(seed)
    shapes = []
    for i in range(count):
        m = int(round(math.exp(rng.uniform(math.log(64), math.log(262144)))))
        n = int(round(math.exp(rng.uniform(math.log(64), math.log(262144)))))
        sigma = int(rng.choice([2, 4, 20, 256]))
        mutated = bool(rng.integers(0, 2))
        batch = int(round(math.exp(rng.uniform(0.0, math.log(4096)))))
        batch = max(1, min(batch, int(cell_cap // (m * n)) or 1))
        shapes.append(Shape(m, n, sigma, mutated, batch, int(rng.integers(0, 2**31 - 1))))
    return shapes


def shape_batch(shape: Shape) -> Batch:
    """Materialise one sweep shape as a batch of `shape.batch` pairs."""
    rng = np.random.default_rng(shape.seed)
    pairs = []
    for _ in range(shape.batch):
        a = uniform(rng, shape.m, shape.sigma)
        if shape.mutated:
            b = fit_length(rng, mutate(rng, a, 0.05, 0.0, 0.0, shape.sigma), shape.n, shape.sigma)
        else:
            b = uniform(rng, shape.n, shape.sigma)
        pairs.append((a, b))
    return pack(pairs)
