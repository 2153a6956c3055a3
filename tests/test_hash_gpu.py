"""PermutationMatrix::hash (src/permutation_matrix.hpp:192-203) of combed
strands computed on the device, for one pair and for every pair of a batch,
against the reference's golden hashes and the host restatement."""
import json
import os

import numpy as np
import pytest

import oracle as O
import slcs
from slcs import workloads as W

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_pair_hash_matches_golden(cuda):
    import torch
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        cases = json.load(f)["test_default"]
    for c in cases:
        a = O.mt19937_binary(c["m"], c["seed_a"]).astype(np.uint8)
        b = O.mt19937_binary(c["n"], c["seed_b"]).astype(np.uint8)
        h, v = slcs.comb_pair(torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda))
        got = slcs.strands_hash(h, v)
        slcs.device_status(0)
        assert got == c["hash"], (c, got)
        assert got == slcs.permutation_hash(O.from_strands(h.cpu().numpy(), v.cpu().numpy())[1])


def test_batch_hashes_match_host(cuda):
    import torch
    rng = np.random.default_rng(21)
    pairs = [(rng.integers(0, 4, int(m), dtype=np.uint8), rng.integers(0, 4, int(n), dtype=np.uint8))
             for m, n in zip(rng.integers(0, 700, 600), rng.integers(0, 900, 600))]
    pairs[3] = (pairs[3][0][:0], pairs[3][1])  # empty sides hash their identity strands
    pairs[7] = (pairs[7][0], pairs[7][1][:0])
    batch = W.pack(pairs)
    off, total = batch.strand_offsets()
    plan = slcs.BatchPlan(slcs.pair_descs(batch))
    out = torch.empty(total, dtype=torch.int32, device=cuda)
    plan.run(torch.from_numpy(batch.a_blob).to(cuda), torch.from_numpy(batch.b_blob).to(cuda), out)
    got = plan.hashes(out).cpu().numpy()
    slcs.device_status(0)
    o = out.cpu().numpy()
    for p in range(batch.npairs):
        m, n = int(batch.ms[p]), int(batch.ns[p])
        h = o[off[p]:off[p] + m]
        v = o[off[p] + m:off[p] + m + n]
        assert int(got[p]) == O.perm_hash(O.from_strands(h, v)[1]), p
    plan.close()
