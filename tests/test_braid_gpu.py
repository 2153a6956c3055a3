"""Parity of the device steady-ant braid multiplication with the oracle's
staggered_multiply (itself pinned to the reference's braid_multiplication.hpp)."""
import numpy as np
import pytest

import oracle as O
import slcs

pytestmark = pytest.mark.gpu


def _dev(x, device):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x, np.int32)).to(device)


def _check(P, Q, k, glue, device, cutoff=None):
    import torch
    want, _ = O.staggered_multiply(P, Q, k, glue)
    got = slcs.braid_multiply(_dev(P, device), _dev(Q, device), k, glue,
                              cfg=slcs.Config.make(braid_cutoff=cutoff) if cutoff else None)
    torch.cuda.synchronize()
    slcs.device_status(0)
    np.testing.assert_array_equal(got.cpu().numpy(), want)


@pytest.mark.parametrize("cutoff", [2, 16, 64, 256, 1024, 4096])
def test_random_permutations(cuda, cutoff):
    rng = np.random.default_rng(cutoff)
    for t in range(40):
        p = int(rng.integers(1, 300)); q = int(rng.integers(1, 300))
        k = int(rng.integers(0, min(p, q) + 1))
        _check(rng.permutation(p), rng.permutation(q), k, bool(t & 1), cuda, cutoff)


@pytest.mark.parametrize("cutoff", [64, 1024, 4096])
def test_comb_composition(cuda, cutoff):
    """P(a, b1) x P(a, b2) with k = m is P(a, b1 b2); row glue likewise."""
    rng = np.random.default_rng(7 + cutoff)
    for t in range(6):
        m, n1, n2 = (int(x) for x in rng.integers(200, 3000, 3))
        a = rng.integers(0, 4, m, dtype=np.uint8)
        b1 = rng.integers(0, 4, n1, dtype=np.uint8)
        b2 = rng.integers(0, 4, n2, dtype=np.uint8)
        P = O.from_strands(*O.comb(a, b1))[0]
        Q = O.from_strands(*O.comb(a, b2))[0]
        _check(P, Q, m, False, cuda, cutoff)
        a2 = rng.integers(0, 4, n2, dtype=np.uint8)
        Q2 = O.from_strands(*O.comb(a2, b1))[0]
        _check(P, Q2, n1, True, cuda, cutoff)


def test_large_merge(cuda):
    rng = np.random.default_rng(3)
    m, n1, n2 = 20000, 9000, 11000
    a = rng.integers(0, 4, m, dtype=np.uint8)
    b1 = rng.integers(0, 4, n1, dtype=np.uint8)
    b2 = rng.integers(0, 4, n2, dtype=np.uint8)
    P = O.from_strands(*O.comb(a, b1))[0]
    Q = O.from_strands(*O.comb(a, b2))[0]
    for cutoff in (256, 4096):
        _check(P, Q, m, False, cuda, cutoff)


@pytest.mark.parametrize("k,cutoff,glue", [(1 << 20, 256, False), (1 << 20, 1024, True), (300001, 256, True),
                                            (600000, 64, False)])
def test_large_random_products(cuda, k, cutoff, glue):
    """Overlaps whose top levels walk in warp segments split into parts
    (grid spacing above 256): power-of-two and other k, both glues."""
    rng = np.random.default_rng(k + cutoff)
    _check(rng.permutation(k + 1000), rng.permutation(k + 3000), k, glue, cuda, cutoff)


def test_small_and_edge_sizes(cuda):
    rng = np.random.default_rng(5)
    for (p, q, k) in [(1, 1, 0), (1, 1, 1), (2, 1, 1), (1, 2, 1), (2, 2, 2), (3, 5, 3), (5, 3, 0), (17, 17, 17)]:
        for glue in (False, True):
            _check(rng.permutation(p), rng.permutation(q), k, glue, cuda)


def test_rejects_non_permutation(cuda):
    import torch
    P = np.array([0, 0, 1], np.int32)
    Q = np.array([2, 1, 0], np.int32)
    slcs.device_status(0)
    slcs.braid_multiply(_dev(P, cuda), _dev(Q, cuda), 2, False)
    torch.cuda.synchronize()
    with pytest.raises(slcs.SlcsError):
        slcs.device_status(0)
