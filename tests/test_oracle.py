"""The oracle pinned against the reference: golden vectors of the reference's own
test script and the reference's code compiled from its sources (oracle/_ref)."""
import json
import os

import numpy as np
import pytest

import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

# test_default.txt of the reference: binary mt19937 strings, seeds 888/999.
TEST_DEFAULT = [(7330, 9944, 944438867), (9771, 11302, 2348829537), (19771, 24302, 3164269182)]


def _ref_or_skip():
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built (reference sources absent)")


def test_golden_hashes_small():
    for (m, n, sa, sb, want) in [(256, 256, 1000, 1001, 4108122986), (4096, 4096, 888, 999, 2010108042),
                                 (7330, 9944, 888, 999, 944438867)]:
        a, b = O.mt19937_binary(m, sa), O.mt19937_binary(n, sb)
        h, v = O.comb(a, b)
        assert O.perm_hash(O.from_strands(h, v)[1]) == want


def test_golden_fixture_file():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        g = json.load(f)
    for case in g["test_default"]:
        a = O.mt19937_binary(case["m"], case["seed_a"])
        b = O.mt19937_binary(case["n"], case["seed_b"])
        if case["m"] * case["n"] > 1.2e8:
            continue  # the largest case is checked on the GPU
        h, v = O.comb(a, b)
        assert O.perm_hash(O.from_strands(h, v)[1]) == case["hash"]


def test_antidiagonal_and_row_orders_agree():
    rng = np.random.default_rng(1)
    for _ in range(50):
        m, n = int(rng.integers(1, 90)), int(rng.integers(1, 90))
        a = rng.integers(0, 3, m, dtype=np.uint8)
        b = rng.integers(0, 3, n, dtype=np.uint8)
        h1, v1 = O.comb(a, b)
        h2, v2 = O.comb_antidiagonal(a, b)
        np.testing.assert_array_equal(h1, h2)
        np.testing.assert_array_equal(v1, v2)


def test_oracle_matches_reference_comb():
    _ref_or_skip()
    rng = np.random.default_rng(2)
    for _ in range(40):
        m, n = int(rng.integers(0, 300)), int(rng.integers(0, 300))
        sigma = int(rng.choice([2, 4, 20, 256]))
        a = rng.integers(0, sigma, m, dtype=np.uint8)
        b = rng.integers(0, sigma, n, dtype=np.uint8)
        h1, v1 = O.comb(a, b)
        h2, v2 = O.ref_comb(a, b)
        np.testing.assert_array_equal(h1, h2)
        np.testing.assert_array_equal(v1, v2)
        r2c, c2r = O.from_strands(h1, v1)
        rh, rc2r = O.ref_hash_from_strands(h2, v2)
        np.testing.assert_array_equal(c2r, rc2r)
        assert O.perm_hash(c2r) == rh


def test_staggered_multiply_matches_reference():
    _ref_or_skip()
    rng = np.random.default_rng(3)
    for t in range(120):
        m, n1, n2 = (int(x) for x in rng.integers(1, 70, 3))
        a = rng.integers(0, 4, m, dtype=np.uint8)
        b1 = rng.integers(0, 4, n1, dtype=np.uint8)
        b2 = rng.integers(0, 4, n2, dtype=np.uint8)
        P = O.from_strands(*O.comb(a, b1))[0]
        Q = O.from_strands(*O.comb(a, b2))[0]
        k = int(rng.integers(0, min(len(P), len(Q)) + 1)) if t % 3 else m
        glue = bool(t & 1)
        r1 = O.staggered_multiply(P, Q, k, glue)
        r2 = O.ref_staggered_multiply(P, Q, k, glue)
        np.testing.assert_array_equal(r1[0], r2[0])
        np.testing.assert_array_equal(r1[1], r2[1])


def test_composition_laws():
    """staggered_multiply<false>(P(a,b1), P(a,b2), m) == P(a, b1|b2) and
    staggered_multiply<true>(P(a1,b), P(a2,b), n) == P(a1|a2, b)."""
    rng = np.random.default_rng(4)
    for _ in range(100):
        m, n1, n2 = (int(x) for x in rng.integers(1, 80, 3))
        sigma = int(rng.choice([2, 4, 256]))
        a = rng.integers(0, sigma, m, dtype=np.uint8)
        a2 = rng.integers(0, sigma, n2, dtype=np.uint8)
        b1 = rng.integers(0, sigma, n1, dtype=np.uint8)
        b2 = rng.integers(0, sigma, n2, dtype=np.uint8)
        P = O.from_strands(*O.comb(a, b1))[0]
        Q = O.from_strands(*O.comb(a, b2))[0]
        R = O.staggered_multiply(P, Q, m, False)[0]
        np.testing.assert_array_equal(R, O.from_strands(*O.comb(a, np.concatenate([b1, b2])))[0])
        P2 = O.from_strands(*O.comb(a, b1))[0]
        Q2 = O.from_strands(*O.comb(a2, b1))[0]
        R2 = O.staggered_multiply(P2, Q2, n1, True)[0]
        np.testing.assert_array_equal(R2, O.from_strands(*O.comb(np.concatenate([a, a2]), b1))[0])


def test_strip_composition_equals_direct():
    rng = np.random.default_rng(5)
    a = rng.integers(0, 4, 3000, dtype=np.uint8)
    b = rng.integers(0, 4, 4100, dtype=np.uint8)
    direct = O.from_strands(*O.comb(a, b))[1]
    for strips in (1, 2, 7, 16):
        np.testing.assert_array_equal(O.comb_strips(a, b, strips, nthreads=4), direct)


def test_tile_composition_equals_direct():
    """Row bands x column strips, glued strips first (overlap = band height)
    and bands second (overlap n), give P(a, b): the algebra of the library's
    tile mode, on uneven bands and strips and with bands of one row."""
    rng = np.random.default_rng(6)
    for m, n, heights, widths in [(300, 200, [100, 100, 100], [50, 150]), (257, 129, [1, 128, 128], [64, 65]),
                                  (64, 300, [64], [16, 16, 268]), (500, 1, [250, 250], [1]),
                                  (333, 444, [32, 1, 300], [100, 44, 300])]:
        sigma = int(rng.choice([2, 4, 20]))
        a = rng.integers(0, sigma, m, dtype=np.uint8)
        b = rng.integers(0, sigma, n, dtype=np.uint8)
        direct = O.from_strands(*O.comb(a, b))[0]
        np.testing.assert_array_equal(O.comb_tiles(a, b, heights, widths), direct)


def test_llcs_identity():
    """LLCS = n - #{j : v[j] >= m} agrees with the classic prefix DP."""
    rng = np.random.default_rng(6)
    for _ in range(60):
        m, n = int(rng.integers(0, 200)), int(rng.integers(0, 200))
        sigma = int(rng.choice([2, 4, 26]))
        a = rng.integers(0, sigma, m, dtype=np.uint8)
        b = rng.integers(0, sigma, n, dtype=np.uint8)
        h, v = O.comb(a, b)
        assert O.llcs_from_strands(h, v) == O.prefix_llcs(a, b)


def test_permutation_is_full():
    rng = np.random.default_rng(7)
    a = rng.integers(0, 4, 500, dtype=np.uint8)
    b = rng.integers(0, 4, 321, dtype=np.uint8)
    r2c, c2r = O.from_strands(*O.comb(a, b))
    assert sorted(r2c.tolist()) == list(range(821))
    np.testing.assert_array_equal(c2r[r2c], np.arange(821))


def test_substring_llcs_formula_matches_dp():
    """LLCS(a, b[i, j)) from the strands equals the DP for every substring."""
    rng = np.random.default_rng(21)
    for _ in range(25):
        m, n = int(rng.integers(1, 30)), int(rng.integers(1, 30))
        s = int(rng.choice([2, 3, 4]))
        a = rng.integers(0, s, m, dtype=np.uint8)
        b = rng.integers(0, s, n, dtype=np.uint8)
        _, v = O.comb(a, b)
        qi, qj = zip(*[(i, j) for i in range(n + 1) for j in range(i, n + 1)])
        got = O.substring_llcs(v, m, qi, qj)
        want = [O.prefix_llcs(a, b[i:j]) if j > i else 0 for i, j in zip(qi, qj)]
        np.testing.assert_array_equal(got, want)
