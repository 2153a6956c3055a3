"""Several GPUs, one process each (torch.distributed; NCCL between GPUs).

Batches of independent pairs shard without any exchange: shard_pairs() deals
the pairs out longest first to the rank with the fewest cells so far, and each
rank combs its shard with its own batch plan.

One long pair splits into G parts, one per rank, either by rows of a (bands)
or by columns of b (strips).  Rank g combs its part, turns the strands into
the part's permutation, and a binary tree of sticky-braid products glues the
parts back together (src/braid_multiplication.hpp:273-407):

    bands:  staggered_multiply<true>(P(x, b), P(y, b), n)  == P(x y, b)
    strips: staggered_multiply<false>(P(a, x), P(a, y), m) == P(a, x y)

In round r, rank g with g % 2^(r+1) == 0 receives the permutation of rank
g + 2^r by point-to-point send/recv -- the peer's array lands in this GPU's
own memory before the product kernel reads it -- and multiplies.  Rank 0 ends
with P(a, b) and returns its strands.  Bands are the default for pairs at
least as tall as they are wide: the stripes of one comb form a chain whose
fill and drain grow with the rows, so G bands of m/G rows each fill G times
faster than G strips of full height (on one B200 the 2^20 x 2^20 pair combs
in 324 ms as 8 bands and 677-729 ms as 8 strips).  Strip widths follow the
library's tile mode (multiples of 16 columns); band heights are whole stripes
of 448 rows (14 rows per lane, the library's choice for the tallest pairs).
Any heights and widths give the same strands.

The compute steps go through a kernels object (CudaKernels: the library's C
ABI) and the exchange through a communicator (TorchComm: torch.distributed
point-to-point on a process group).  The exchange logic depends on neither,
which is how it is tested on CPU processes with the gloo backend and, with
in-process ranks that hand tensors over by device copies, through the CUDA
kernels on one GPU.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence, Tuple

import numpy as np


def strip_widths(n: int, strips: int) -> List[int]:
    """Widths of `strips` column strips of n columns, left to right: each a
    multiple of 16 (at least 16) while columns last, the last strip takes the
    rest; strips past the end of b are empty."""
    strips = max(1, int(strips))
    base = max(16, n // strips // 16 * 16)
    out, left = [], n
    for s in range(strips):
        w = min(base, left) if s + 1 < strips else left
        out.append(w)
        left -= w
    return out


def band_heights(m: int, bands: int, rows_per_stripe: int = 448) -> List[int]:
    """Heights of `bands` row bands of m rows, top to bottom: whole stripes of
    `rows_per_stripe` rows, as equal in stripes as the stripe count allows;
    the last band takes the rest."""
    bands = max(1, int(bands))
    stripes = (m + rows_per_stripe - 1) // rows_per_stripe if m > 0 else 0
    out, left = [], m
    for r in range(bands):
        want = (stripes * (r + 1) // bands - stripes * r // bands) * rows_per_stripe
        h = min(want, left) if r + 1 < bands else left
        out.append(h)
        left -= h
    return out


def shard_pairs(cells: Sequence[int], world: int) -> List[np.ndarray]:
    """Pair indices per rank: largest first to the least loaded rank (LPT)."""
    cells = np.asarray(cells, np.int64)
    order = np.argsort(-cells, kind="stable")
    heap = [(0, r) for r in range(world)]
    shards: List[list] = [[] for _ in range(world)]
    for p in order:
        load, r = heapq.heappop(heap)
        shards[r].append(int(p))
        heapq.heappush(heap, (load + int(cells[p]), r))
    return [np.array(sorted(s), np.int64) for s in shards]


def merge_rounds(world: int) -> List[List[Tuple[int, int]]]:
    """Rounds of the merge tree: (receiver, sender) pairs; the receiver's
    strips lie left of the sender's."""
    rounds, step = [], 1
    while step < world:
        rounds.append([(g, g + step) for g in range(0, world, 2 * step) if g + step < world])
        step *= 2
    return rounds


class CudaKernels:
    """The library's GPU entry points on torch CUDA tensors."""

    def __init__(self, cfg=None):
        self.cfg = cfg

    def comb(self, a, b):
        from . import comb_pair
        return comb_pair(a, b, cfg=self.cfg)

    def to_perm(self, h, v):
        from . import strands_to_permutation
        return strands_to_permutation(h, v)[0]

    def braid(self, p, q, k, row_glue=False):
        from . import braid_multiply
        return braid_multiply(p, q, k, row_glue, cfg=self.cfg)

    def to_strands(self, r2c, m):
        from . import permutation_to_strands
        return permutation_to_strands(r2c, m)

    def empty(self, size, like):
        import torch
        return torch.empty(int(size), dtype=torch.int32, device=like.device)


class TorchComm:
    """Point-to-point exchange over a torch.distributed process group (NCCL
    between GPUs, gloo between CPU processes)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def send(self, t, dst: int):
        import torch.distributed as dist
        dist.send(t, group=self.group, group_dst=dst)

    def recv(self, t, src: int):
        import torch.distributed as dist
        dist.recv(t, group=self.group, group_src=src)


def comb_pair_distributed(a, b, group=None, kernels=None, split: str = "auto", comm=None):
    """Strands (h, v) of one pair on rank 0 (None on the other ranks).

    a and b are the whole strings on every rank (uint8 tensors on this rank's
    device); each rank reads only its band of a or strip of b.  split is
    "bands", "strips" or "auto" (bands when m >= n).  Every rank takes the
    same send/recv steps in the same order.  `comm` (rank, world, send,
    recv) defaults to TorchComm(group)."""
    K = kernels or CudaKernels()
    C = comm or TorchComm(group)
    rank, world = C.rank, C.world
    m, n = int(a.numel()), int(b.numel())
    if split == "auto":
        split = "bands" if m >= n else "strips"
    if split not in ("bands", "strips"):
        raise ValueError("split must be 'bands', 'strips' or 'auto'")
    rows = split == "bands"
    parts = band_heights(m, world) if rows else strip_widths(n, world)
    start = sum(parts[:rank])
    if rows:
        h, v = K.comb(a[start:start + parts[rank]], b)
    else:
        h, v = K.comb(a, b[start:start + parts[rank]])
    P = K.to_perm(h, v)
    k = n if rows else m  # overlap of every product
    sizes = [p + k for p in parts]  # current permutation size held by each rank
    for rnd in merge_rounds(world):
        for dst, src in rnd:
            if rank == src:
                C.send(P, dst)
            elif rank == dst:
                Q = K.empty(sizes[src], P)
                C.recv(Q, src)
                P = K.braid(P, Q, k, rows)
        for dst, src in rnd:
            sizes[dst] = sizes[dst] + sizes[src] - k
    if rank != 0:
        return None
    return K.to_strands(P, m)
