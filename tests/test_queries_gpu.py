"""Semi-local string-substring LCS from the strands on the GPU
(slcs_substring_llcs) against the oracle's formula and the DP."""
import numpy as np
import pytest

import oracle as O
import slcs

pytestmark = pytest.mark.gpu


def _dev(x, device):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(device)


def test_every_substring_small(cuda):
    rng = np.random.default_rng(31)
    for _ in range(10):
        m, n = int(rng.integers(1, 60)), int(rng.integers(1, 90))
        a = rng.integers(0, 3, m, dtype=np.uint8)
        b = rng.integers(0, 3, n, dtype=np.uint8)
        _, v = slcs.comb_pair(_dev(a, cuda), _dev(b, cuda))
        qi, qj = map(np.array, zip(*[(i, j) for i in range(n + 1) for j in range(i, n + 1)]))
        got = slcs.substring_llcs(v, m, _dev(qi.astype(np.int32), cuda), _dev(qj.astype(np.int32), cuda))
        want = [O.prefix_llcs(a, b[i:j]) if j > i else 0 for i, j in zip(qi, qj)]
        np.testing.assert_array_equal(got.cpu().numpy(), want)


def test_many_queries_long_pair(cuda):
    """Random substrings of a 3000 x 200000 pair against the formula on the
    oracle's strands, a few against the DP."""
    rng = np.random.default_rng(32)
    m, n = 3000, 200000
    a = rng.integers(0, 4, m, dtype=np.uint8)
    b = rng.integers(0, 4, n, dtype=np.uint8)
    _, v = slcs.comb_pair(_dev(a, cuda), _dev(b, cuda))
    _, ev = O.comb(a, b)
    np.testing.assert_array_equal(v.cpu().numpy(), ev)
    qi = rng.integers(0, n, 5000).astype(np.int32)
    qj = np.minimum(n, qi + rng.integers(0, 20000, 5000)).astype(np.int32)
    got = slcs.substring_llcs(v, m, _dev(qi, cuda), _dev(qj, cuda)).cpu().numpy()
    np.testing.assert_array_equal(got, O.substring_llcs(ev, m, qi, qj))
    for q in range(3):
        assert got[q] == O.prefix_llcs(a, b[qi[q]:qj[q]])


def test_bad_query_reports_invalid(cuda):
    rng = np.random.default_rng(33)
    a = rng.integers(0, 4, 50, dtype=np.uint8)
    b = rng.integers(0, 4, 80, dtype=np.uint8)
    _, v = slcs.comb_pair(_dev(a, cuda), _dev(b, cuda))
    qi = np.array([0, 10, 70], np.int32)
    qj = np.array([80, 5, 90], np.int32)  # second: end < begin; third: end > n
    got = slcs.substring_llcs(v, 50, _dev(qi, cuda), _dev(qj, cuda)).cpu().numpy()
    assert got[0] == O.prefix_llcs(a, b) and got[1] == -1 and got[2] == -1
    with pytest.raises(slcs.SlcsError):
        slcs.device_status(0)
    slcs.device_status(0)  # the first check cleared the bit
