"""The reference-side procedure adapter (Lcs_Semi_B200 behind the C++ mirror
of LcsAlgorithmRegistry) on Word symbols of any value: the symbols become
bytes on the device (slcs_symbols_to_bytes), the strands must equal the
oracle's comb of the original int32 symbols (src/lcs_residual_fixup.hpp:4-70
compares Words for equality only), length_of_lcs must equal the LCS length,
and more than 256 distinct symbols must raise the adapter's exception."""
import numpy as np
import pytest

import oracle as O
import slcs

pytestmark = pytest.mark.gpu


def _words(rng, alphabet, m, n):
    return rng.choice(alphabet, m).astype(np.int32), rng.choice(alphabet, n).astype(np.int32)


def _ranks(a, b):
    u = np.unique(np.concatenate([a, b]))
    return np.searchsorted(u, a).astype(np.uint8), np.searchsorted(u, b).astype(np.uint8)


@pytest.mark.parametrize("kind", ["negative", "wide", "bytes", "max256"])
def test_procedure_on_word_symbols(cuda, kind):
    rng = np.random.default_rng({"negative": 1, "wide": 2, "bytes": 3, "max256": 4}[kind])
    if kind == "negative":
        alphabet = np.array([-7, -1, 0, 3, 1 << 30], np.int64)
    elif kind == "wide":
        alphabet = rng.choice(np.arange(-(1 << 31), (1 << 31) - 1, 7919, dtype=np.int64), 40, replace=False)
    elif kind == "bytes":
        alphabet = np.arange(0, 256, 9)
    else:
        alphabet = np.arange(256, dtype=np.int64) * 1000003 - (1 << 27)
    a, b = _words(rng, alphabet, 1500, 1777)
    if kind == "max256":
        a[:256] = alphabet  # every one of the 256 symbols occurs
    for name in ("b200", "b200_4_4", "b200_strips_4_1024"):
        rc, h, v, llcs, hv, msg = slcs.run_procedure(name, a, b)
        assert rc == 0, msg
        eh, ev = O.comb_antidiagonal(a, b)
        assert np.array_equal(h, eh) and np.array_equal(v, ev), name
        ar, br = _ranks(a, b)
        assert llcs == O.prefix_llcs(ar, br) == O.llcs_from_strands(eh, ev)
        assert hv == O.perm_hash(O.from_strands(eh, ev)[1])


def test_more_than_256_symbols_raise(cuda):
    rng = np.random.default_rng(9)
    a = np.arange(257, dtype=np.int32) * 3 - 100
    b = rng.choice(a, 300).astype(np.int32)
    rc, _, _, _, _, msg = slcs.run_procedure("b200", a, b)
    assert rc == 2 and "256" in msg
    with pytest.raises(slcs.SlcsError) as err:
        slcs.comb_pair_words_host(a, b)
    assert err.value.status == 6


def test_symbols_to_bytes_on_device(cuda):
    import torch
    rng = np.random.default_rng(11)
    for alphabet in (np.array([5, 200, 17]), np.array([-3, 99999, 4, -(1 << 31), (1 << 31) - 1])):
        a, b = _words(rng, alphabet, 70000, 50001)
        ab, bb, k = slcs.symbols_to_bytes(torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda))
        torch.cuda.synchronize()
        want = (a.astype(np.uint8), b.astype(np.uint8)) if alphabet.min() >= 0 and alphabet.max() < 256 \
            else _ranks(a, b)
        assert k == len(np.unique(np.concatenate([a, b])))
        assert np.array_equal(ab.cpu().numpy(), want[0]) and np.array_equal(bb.cpu().numpy(), want[1])
    # empty sides and a large alphabet spread over many blocks
    big = np.arange(100000, dtype=np.int32)
    _, _, k = slcs.symbols_to_bytes(torch.from_numpy(big).to(cuda), torch.from_numpy(big[:0]).to(cuda))
    assert k == -1
    _, _, k = slcs.symbols_to_bytes(torch.from_numpy(big[:0]).to(cuda), torch.from_numpy(big[:0]).to(cuda))
    assert k == 0


def test_words_host_entry_matches_byte_entry(cuda):
    rng = np.random.default_rng(12)
    a = rng.integers(0, 4, 3000).astype(np.int32) * 1000 - 1500
    b = rng.integers(0, 4, 2000).astype(np.int32) * 1000 - 1500
    h, v = slcs.comb_pair_words_host(a, b)
    ar, br = _ranks(a, b)
    eh, ev = slcs.comb_pair_host(ar, br)
    assert np.array_equal(h, eh) and np.array_equal(v, ev)
