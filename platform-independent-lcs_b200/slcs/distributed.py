"""Several GPUs, one process each (torch.distributed; NCCL between GPUs).

Batches of independent pairs shard without any exchange: shard_pairs() deals
the pairs out longest first to the rank with the fewest cells so far, and each
rank combs its shard with its own batch plan.

One long pair splits by columns of b.  Rank g combs the strip (a, b_g), turns
its strands into the permutation P(a, b_g), and a binary tree of sticky-braid
products with overlap m glues the strips back together
(staggered_multiply<false>(P(a, x), P(a, y), m) == P(a, x y),
src/braid_multiplication.hpp:273-407): in round r, rank g with
g % 2^(r+1) == 0 receives the permutation of rank g + 2^r by point-to-point
send/recv -- the peer's array lands in this GPU's own memory before the
product kernel reads it -- and multiplies.  Rank 0 ends with P(a, b) and
returns its strands.  Strip widths follow the library's strip mode, so one
GPU in strip mode and G GPUs produce the same products.

The compute steps go through a kernels object (CudaKernels: the library's C
ABI).  The exchange logic does not depend on what computes, which is how it
is tested on CPU processes with the gloo backend.
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

    def braid(self, p, q, k):
        from . import braid_multiply
        return braid_multiply(p, q, k, False, cfg=self.cfg)

    def to_strands(self, r2c, m):
        from . import permutation_to_strands
        return permutation_to_strands(r2c, m)

    def empty(self, size, like):
        import torch
        return torch.empty(int(size), dtype=torch.int32, device=like.device)


def comb_pair_distributed(a, b, group=None, kernels=None):
    """Strands (h, v) of one pair on rank 0 (None on the other ranks).

    a and b are the whole strings on every rank (uint8 tensors on this rank's
    device); each rank reads only its strip of b.  Every rank takes the same
    send/recv steps in the same order."""
    import torch.distributed as dist
    K = kernels or CudaKernels()
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    m, n = int(a.numel()), int(b.numel())
    widths = strip_widths(n, world)
    start = sum(widths[:rank])
    h, v = K.comb(a, b[start:start + widths[rank]])
    P = K.to_perm(h, v)
    sizes = [m + w for w in widths]  # current permutation size held by each rank
    for rnd in merge_rounds(world):
        for dst, src in rnd:
            if rank == src:
                dist.send(P, group=group, group_dst=dst)
            elif rank == dst:
                Q = K.empty(sizes[src], P)
                dist.recv(Q, group=group, group_src=src)
                P = K.braid(P, Q, m)
        for dst, src in rnd:
            sizes[dst] = sizes[dst] + sizes[src] - m
    if rank != 0:
        return None
    return K.to_strands(P, m)
