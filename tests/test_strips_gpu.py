"""Strip mode: one pair combed as column strips and glued by steady-ant braid
multiplication (staggered_multiply<false> with overlap m) must return exactly
the strands of the direct comb."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle as O
import slcs
from slcs import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.json")


def _dev(x, device):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(device)


@pytest.mark.parametrize("m,n,strips,cutoff", [(1, 200, 3, 0), (300, 64, 8, 0), (1000, 1500, 2, 64),
                                               (777, 4099, 5, 256), (2049, 3001, 8, 1024), (4096, 4096, 7, 4096),
                                               (5000, 130, 2, 0)])
def test_strips_match_direct_comb(cuda, m, n, strips, cutoff):
    rng = np.random.default_rng(m * 7 + n)
    sigma = int(rng.choice([2, 4, 20]))
    a = rng.integers(0, sigma, m, dtype=np.uint8)
    b = rng.integers(0, sigma, n, dtype=np.uint8)
    cfg = slcs.Config.make(algo=slcs.ALGO_STRIPS, strips=strips, braid_cutoff=cutoff or None)
    h, v = slcs.comb_pair(_dev(a, cuda), _dev(b, cuda), cfg=cfg)
    slcs.device_status(0)
    eh, ev = O.comb(a, b)
    np.testing.assert_array_equal(h.cpu().numpy(), eh)
    np.testing.assert_array_equal(v.cpu().numpy(), ev)


def _golden(name):
    with open(GOLDEN) as f:
        return json.load(f)[name]


@pytest.mark.parametrize("cutoff", [64, 256, 1024, 4096])
def test_strips_pair_1m_cutoff_sweep(cuda, cutoff):
    """The 2^20 x 2^20 pair as 8 strips merged with every braid cutoff of the sweep."""
    g = _golden("pair_1M")
    a, b = W.pair_1m()
    cfg = slcs.Config.make(algo=slcs.ALGO_STRIPS, strips=8, braid_cutoff=cutoff)
    h, v = slcs.comb_pair(_dev(a, cuda), _dev(b, cuda), cfg=cfg)
    _, c2r = slcs.strands_to_permutation(h, v)
    c2r = c2r.cpu().numpy()
    slcs.device_status(0)
    assert hashlib.sha256(c2r.tobytes()).hexdigest() == g["sha256_col_to_row"]


def test_strips_pair_131072_mutated(cuda):
    g = _golden("pair_131072_mutated")
    a, b = W.pair_131072_mutated()
    cfg = slcs.Config.make(algo=slcs.ALGO_STRIPS, strips=16)
    h, v = slcs.comb_pair(_dev(a, cuda), _dev(b, cuda), cfg=cfg)
    _, c2r = slcs.strands_to_permutation(h, v)
    c2r = c2r.cpu().numpy()
    assert hashlib.sha256(c2r.tobytes()).hexdigest() == g["sha256_col_to_row"]
    assert slcs.permutation_hash(c2r) == g["hash"]


@pytest.mark.parametrize("m,n", [(600, 300000), (20000, 70000), (5000, 5000)])
def test_default_rule_picks_strips_and_matches(cuda, m, n):
    """The default configuration combs wide and mid-size pairs as strips
    (many strips for a short, wide pair); strands equal the oracle's."""
    rng = np.random.default_rng(m + n)
    a = rng.integers(0, 4, m, dtype=np.uint8)
    b = rng.integers(0, 4, n, dtype=np.uint8)
    h, v = slcs.comb_pair(_dev(a, cuda), _dev(b, cuda))
    slcs.device_status(0)
    eh, ev = O.comb(a, b)
    np.testing.assert_array_equal(h.cpu().numpy(), eh)
    np.testing.assert_array_equal(v.cpu().numpy(), ev)
