"""Tile mode: one pair combed as row bands x column strips and glued by
steady-ant braid multiplication (staggered_multiply<false> with overlap = band
height across strips, staggered_multiply<true> with overlap n across bands)
must return exactly the strands of the direct comb."""
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


@pytest.mark.parametrize("m,n,bands,strips,tm,cutoff", [
    (3000, 2000, 2, 1, 4, 0), (5000, 1500, 3, 2, 8, 64), (4097, 333, 5, 1, 2, 256),
    (64, 5000, 4, 3, 2, 0), (10000, 1, 4, 1, 4, 0), (7000, 7000, 16, 2, 14, 1024), (1, 1, 2, 2, 2, 0),
    (20000, 10007, 8, 1, 16, 0)])
def test_bands_match_direct_comb(cuda, m, n, bands, strips, tm, cutoff):
    """Row bands (whole stripes of 32*tm rows; more bands than stripes are
    capped) and strips together, including n = 1 (row-glue overlap 1) and
    tiles short enough against their width for 8 columns per step (7000^2 in
    16 x 2 tiles, 20000 x 10007 in 8 bands: ragged last block)."""
    rng = np.random.default_rng(m * 3 + n + bands)
    sigma = int(rng.choice([2, 4, 20]))
    a = rng.integers(0, sigma, m, dtype=np.uint8)
    b = rng.integers(0, sigma, n, dtype=np.uint8)
    cfg = slcs.Config.make(algo=slcs.ALGO_STRIPS, strips=strips, bands=bands, tile_m=tm,
                           braid_cutoff=cutoff or None)
    h, v = slcs.comb_pair(_dev(a, cuda), _dev(b, cuda), cfg=cfg)
    slcs.device_status(0)
    eh, ev = O.comb(a, b)
    np.testing.assert_array_equal(h.cpu().numpy(), eh)
    np.testing.assert_array_equal(v.cpu().numpy(), ev)


def test_default_rule_picks_bands_for_tall_pairs(cuda):
    """Pairs of 2^19 rows and more: the default combs them in row bands (a
    narrow pair in many, since its stripe chain is long against its width)."""
    info = slcs.pair_plan_info(1 << 20, 1 << 20)
    assert info["algo"] == slcs.ALGO_STRIPS and info["bands"] > 1 and info["strips"] == 1
    m, n = (1 << 19) + 77, 700
    info = slcs.pair_plan_info(m, n)
    assert info["bands"] >= 8
    rng = np.random.default_rng(19)
    a = rng.integers(0, 4, m, dtype=np.uint8)
    b = rng.integers(0, 4, n, dtype=np.uint8)
    h, v = slcs.comb_pair(_dev(a, cuda), _dev(b, cuda))
    slcs.device_status(0)
    eh, ev = O.comb(a, b)
    np.testing.assert_array_equal(h.cpu().numpy(), eh)
    np.testing.assert_array_equal(v.cpu().numpy(), ev)


def test_pair_plan_info_follows_config(cuda):
    assert slcs.pair_plan_info(0, 5)["algo"] == 0
    info = slcs.pair_plan_info(3000, 3000, slcs.Config.make(algo=1, tile_m=8, warps=2))
    assert (info["algo"], info["tile_m"], info["warps"], info["strips"], info["bands"]) == (1, 8, 2, 1, 1)
    assert info["stripes"] == (3000 + 255) // 256
    info = slcs.pair_plan_info(3000, 3000, slcs.Config.make(algo=2, strips=3, bands=2, tile_m=4))
    assert (info["algo"], info["strips"], info["bands"], info["braid_cutoff"]) == (2, 3, 2, 1024)
