"""The multi-GPU split of one long pair, driven through the CUDA kernels on one
GPU: every rank of the merge tree (comb of its band or strip,
strands_to_permutation, braid products in tree order, permutation_to_strands
on rank 0) runs as a thread of this process, and the point-to-point exchange
is a device copy into the receiver's own buffer.  The ranks' kernels never
wait on one another: a receiver blocks on the host until the sender's tensor
has been enqueued, and all work is ordered on one stream.  The strands of
rank 0 must equal the CPU oracle's comb of the whole pair
(src/braid_multiplication.hpp:273-407 glues the parts)."""
import queue
import threading

import numpy as np
import pytest

import oracle as O
from slcs import distributed as D

pytestmark = pytest.mark.gpu


class ThreadComm:
    """In-process ranks: send enqueues a device copy of the tensor, recv copies
    it into the receiver's buffer."""

    def __init__(self, rank, world, boxes):
        self.rank, self.world, self.boxes = rank, world, boxes

    def send(self, t, dst):
        self.boxes[(self.rank, dst)].put(t.clone())

    def recv(self, t, src):
        t.copy_(self.boxes[(src, self.rank)].get(timeout=120))


def _run_ranks(a, b, world, split, cuda):
    import torch
    boxes = {(s, d): queue.Queue() for s in range(world) for d in range(world)}
    results, errors = [None] * world, []

    def rank_main(r):
        try:
            torch.cuda.set_device(cuda)
            ad = torch.from_numpy(a).to(cuda)
            bd = torch.from_numpy(b).to(cuda)
            results[r] = D.comb_pair_distributed(ad, bd, kernels=D.CudaKernels(), split=split,
                                                 comm=ThreadComm(r, world, boxes))
            torch.cuda.synchronize()
        except Exception as e:  # reported by the test below
            errors.append((r, repr(e)))

    threads = [threading.Thread(target=rank_main, args=(r,)) for r in range(world)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in threads), "a rank did not finish"
    assert not errors, errors
    assert all(x is None for x in results[1:])
    return results[0]


@pytest.mark.parametrize("world", [2, 3, 8])
@pytest.mark.parametrize("split,m,n", [("bands", 4000, 3000), ("strips", 2500, 3900)])
def test_distributed_pair_on_cuda_kernels(cuda, world, split, m, n):
    import slcs
    rng = np.random.default_rng(100 * world + len(split))
    a = rng.integers(0, 4, m, dtype=np.uint8)
    b = rng.integers(0, 4, n, dtype=np.uint8)
    h, v = _run_ranks(a, b, world, split, cuda)
    slcs.device_status(0)
    eh, ev = O.comb(a, b)
    assert np.array_equal(h.cpu().numpy(), eh)
    assert np.array_equal(v.cpu().numpy(), ev)


def test_distributed_auto_split_mutated_pair(cuda):
    """split="auto" on a tall mutated pair (bands) and a wide one (strips)."""
    import slcs
    from slcs import workloads as W
    rng = np.random.default_rng(5)
    a = W.uniform(rng, 6000)
    b = W.fit_length(rng, W.mutate(rng, a, 0.1, 0.01, 0.01), 5000)
    for x, y in ((a, b), (b, a)):
        h, v = _run_ranks(x, y, 4, "auto", cuda)
        slcs.device_status(0)
        eh, ev = O.comb(x, y)
        assert np.array_equal(h.cpu().numpy(), eh) and np.array_equal(v.cpu().numpy(), ev)
