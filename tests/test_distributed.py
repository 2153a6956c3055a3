"""The multi-GPU split on CPU processes (gloo, world sizes 2 and 3): strip
widths, the merge schedule, LPT sharding, and the send/recv merge tree of one
long pair, with the compute steps done by the CPU oracle so that the exchange
logic is checked without a GPU."""
import os
import tempfile

import numpy as np
import pytest

import oracle as O
from slcs import distributed as D

HERE = os.path.dirname(os.path.abspath(__file__))


def test_strip_widths():
    for n in (0, 1, 15, 16, 100, 4096, 131072, 1000003):
        for s in (1, 2, 3, 8):
            w = D.strip_widths(n, s)
            assert len(w) == s and sum(w) == n and min(w) >= 0
            assert all(w[i] % 16 == 0 or sum(w[i + 1:]) == 0 for i in range(s - 1))


def test_band_heights():
    for m in (0, 1, 447, 448, 449, 5000, 1 << 20):
        for bands in (1, 2, 3, 8):
            h = D.band_heights(m, bands)
            assert len(h) == bands and sum(h) == m and min(h) >= 0
            assert all(x % 448 == 0 for x in h[:-1])


def test_merge_rounds_cover_every_rank_once():
    for world in range(1, 9):
        alive = set(range(world))
        for rnd in D.merge_rounds(world):
            for dst, src in rnd:
                assert dst in alive and src in alive and dst < src
                alive.discard(src)
        assert alive == {0}


def test_shard_pairs_lpt():
    rng = np.random.default_rng(3)
    cells = rng.integers(1, 10**6, 5000)
    for world in (1, 2, 3, 8):
        shards = D.shard_pairs(cells, world)
        assert sorted(np.concatenate(shards).tolist()) == list(range(len(cells)))
        loads = [int(cells[s].sum()) for s in shards]
        assert max(loads) - min(loads) <= int(cells.max())


class OracleKernels:
    """CPU stand-ins for the compute steps (torch CPU tensors)."""

    def comb(self, a, b):
        import torch
        h, v = O.comb(a.numpy(), b.numpy())
        return torch.from_numpy(h), torch.from_numpy(v)

    def to_perm(self, h, v):
        import torch
        return torch.from_numpy(O.from_strands(h.numpy(), v.numpy())[0])

    def braid(self, p, q, k, row_glue=False):
        import torch
        return torch.from_numpy(O.staggered_multiply(p.numpy(), q.numpy(), k, row_glue)[0])

    def to_strands(self, r2c, m):
        import torch
        r = r2c.numpy()
        n = len(r) - m
        h = np.empty(m, np.int32)
        v = np.empty(n, np.int32)
        rows = np.arange(len(r), dtype=np.int32)
        v[r[r < n]] = rows[r < n]
        h[r[r >= n] - n] = rows[r >= n]
        return torch.from_numpy(h), torch.from_numpy(v)

    def empty(self, size, like):
        import torch
        return torch.empty(int(size), dtype=torch.int32)


def _worker(rank, world, port, m, n, seed, out_path, split):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(seed)
        a = torch.from_numpy(rng.integers(0, 4, m, dtype=np.uint8))
        b = torch.from_numpy(rng.integers(0, 4, n, dtype=np.uint8))
        res = D.comb_pair_distributed(a, b, kernels=OracleKernels(), split=split)
        if rank == 0:
            np.savez(out_path, h=res[0].numpy(), v=res[1].numpy())
        else:
            assert res is None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,m,n,split", [(2, 300, 1000, "strips"), (3, 257, 777, "strips"), (2, 100, 20, "auto"),
                                             (2, 1000, 300, "bands"), (3, 1500, 257, "auto"), (2, 5, 40, "bands")])
def test_comb_pair_distributed_gloo(world, m, n, split):
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    seed = 17 + world + m
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "res.npz")
        mp.start_processes(_worker, args=(world, port, m, n, seed, out, split), nprocs=world, join=True,
                           start_method="spawn")
        got = np.load(out)
        rng = np.random.default_rng(seed)
        a = rng.integers(0, 4, m, dtype=np.uint8)
        b = rng.integers(0, 4, n, dtype=np.uint8)
        eh, ev = O.comb(a, b)
        np.testing.assert_array_equal(got["h"], eh)
        np.testing.assert_array_equal(got["v"], ev)


def _worker_fail(rank, world, port, out_dir):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        if rank == 1:
            raise RuntimeError("rank 1 failed before its send")  # the failure, made on the host
        rng = np.random.default_rng(3)
        a = torch.from_numpy(rng.integers(0, 4, 200, dtype=np.uint8))
        b = torch.from_numpy(rng.integers(0, 4, 500, dtype=np.uint8))
        try:
            D.comb_pair_distributed(a, b, kernels=OracleKernels(), split="strips")
            open(os.path.join(out_dir, "rank0_finished"), "w").close()
        except Exception as e:  # the receive from the failed rank ends in an error
            with open(os.path.join(out_dir, "rank0_error"), "w") as f:
                f.write(repr(e))
    finally:
        dist.destroy_process_group()


def test_failed_rank_ends_the_merge_with_an_error():
    """A rank that fails before its send: the receiving rank's point-to-point
    receive ends with an error (peer gone or the group's 10 s timeout)
    instead of waiting for good; no GPU is involved."""
    import socket
    import time

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    with tempfile.TemporaryDirectory() as d:
        ctx = mp.start_processes(_worker_fail, args=(2, port, d), nprocs=2, join=False, start_method="spawn")
        deadline = time.time() + 120
        for p in ctx.processes:
            p.join(timeout=max(1.0, deadline - time.time()))
        alive = [p for p in ctx.processes if p.is_alive()]
        for p in alive:
            p.kill()
        assert not alive, "a rank was still waiting"
        assert ctx.processes[1].exitcode != 0
        assert os.path.exists(os.path.join(d, "rank0_error"))
        assert not os.path.exists(os.path.join(d, "rank0_finished"))
