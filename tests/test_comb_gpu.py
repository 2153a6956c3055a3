"""Parity of the CUDA combing kernels with the CPU oracle (bit-exact strands)."""
import numpy as np
import pytest

import oracle as O
import slcs
from slcs import workloads as W

pytestmark = pytest.mark.gpu


def _dev(x, device):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x)).to(device)


def _check_pair(a, b, device, cfg=None):
    h, v = slcs.comb_pair(_dev(a, device), _dev(b, device), cfg=cfg)
    import torch
    torch.cuda.synchronize()
    slcs.device_status(0)
    eh, ev = O.comb(a, b)
    np.testing.assert_array_equal(h.cpu().numpy(), eh)
    np.testing.assert_array_equal(v.cpu().numpy(), ev)


SHAPES = [(1, 1), (1, 7), (7, 1), (2, 3), (31, 33), (32, 32), (33, 4), (64, 129), (127, 255),
          (257, 100), (500, 3), (3, 500), (1000, 1001), (1023, 517), (2049, 2047)]


@pytest.mark.parametrize("tm", [2, 4, 8, 12, 14, 16])
def test_pair_shapes(cuda, tm):
    rng = np.random.default_rng(10 + tm)
    for (m, n) in SHAPES:
        sigma = int(rng.choice([2, 4, 20, 256]))
        a = rng.integers(0, sigma, m, dtype=np.uint8)
        b = rng.integers(0, sigma, n, dtype=np.uint8)
        _check_pair(a, b, cuda, slcs.Config.make(tile_m=tm))


@pytest.mark.parametrize("tm,m,n", [(2, 160000, 333), (14, 7 * 448 + 5, 1001), (16, 64 * 512 + 1, 97),
                                    (16, 1000, 9001), (14, 900, 6007)])
def test_pair_stripe_counts(cuda, tm, m, n):
    """Stripe counts around the resident capacity: 2500 stripes of 64 rows are
    more than one launch holds at once (persistent blocks take stripes from the
    ticket counter); the others run one block per SM, the last one with a
    single-row stripe at the bottom; the last two are short chains against
    their width, combed 8 columns per step (ragged last block)."""
    rng = np.random.default_rng(m + n)
    a = rng.integers(0, 4, m, dtype=np.uint8)
    b = rng.integers(0, 4, n, dtype=np.uint8)
    _check_pair(a, b, cuda, slcs.Config.make(tile_m=tm))


@pytest.mark.parametrize("warps", [2, 4, 8])
def test_pair_warps(cuda, warps):
    rng = np.random.default_rng(warps)
    a = rng.integers(0, 4, 3000, dtype=np.uint8)
    b = rng.integers(0, 4, 2500, dtype=np.uint8)
    _check_pair(a, b, cuda, slcs.Config.make(tile_m=2, warps=warps))


def test_pair_4096_golden(cuda):
    a, b = W.pair_4096()
    h, v = slcs.comb_pair(_dev(a, cuda), _dev(b, cuda))
    r2c, c2r = slcs.strands_to_permutation(h, v)
    c2r = c2r.cpu().numpy()
    eh, ev = O.comb(a, b)
    er2c, ec2r = O.from_strands(eh, ev)
    np.testing.assert_array_equal(c2r, ec2r)
    np.testing.assert_array_equal(r2c.cpu().numpy(), er2c)
    assert slcs.permutation_hash(c2r) == O.perm_hash(ec2r)


def test_test_default_hashes(cuda):
    """The reference's own test script cases (test_default.txt) by hash."""
    for (m, n, want) in [(7330, 9944, 944438867), (9771, 11302, 2348829537), (19771, 24302, 3164269182)]:
        a = O.mt19937_binary(m, 888)
        b = O.mt19937_binary(n, 999)
        h, v = slcs.comb_pair(_dev(a, cuda), _dev(b, cuda))
        _, c2r = slcs.strands_to_permutation(h, v)
        assert slcs.permutation_hash(c2r.cpu().numpy()) == want


def test_pair_unaligned_and_split_outputs(cuda):
    import torch
    rng = np.random.default_rng(3)
    a = rng.integers(0, 4, 777, dtype=np.uint8)
    b = rng.integers(0, 4, 901, dtype=np.uint8)
    abuf = _dev(np.concatenate([[9], a]).astype(np.uint8), cuda)
    bbuf = _dev(np.concatenate([[9, 9, 9], b]).astype(np.uint8), cuda)
    h = torch.empty(777, dtype=torch.int32, device=cuda)
    v = torch.empty(901, dtype=torch.int32, device=cuda)
    L = slcs.lib()
    slcs.check(L.slcs_comb_pair(abuf.data_ptr() + 1, 777, bbuf.data_ptr() + 3, 901, h.data_ptr(), v.data_ptr(),
                                None, torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    eh, ev = O.comb(a, b)
    np.testing.assert_array_equal(h.cpu().numpy(), eh)
    np.testing.assert_array_equal(v.cpu().numpy(), ev)


def test_pair_empty_sides(cuda):
    for (m, n) in [(0, 5), (5, 0), (0, 0)]:
        h, v = slcs.comb_pair_host(np.zeros(m, np.uint8), np.zeros(n, np.uint8))
        np.testing.assert_array_equal(h, np.arange(m))
        np.testing.assert_array_equal(v, np.arange(m, m + n))


def test_pair_host_api(cuda):
    rng = np.random.default_rng(4)
    a = rng.integers(0, 20, 1500, dtype=np.uint8)
    b = rng.integers(0, 20, 1700, dtype=np.uint8)
    h, v = slcs.comb_pair_host(a, b)
    eh, ev = O.comb(a, b)
    np.testing.assert_array_equal(h, eh)
    np.testing.assert_array_equal(v, ev)


def _batch_expected(batch):
    off, total = batch.strand_offsets()
    return O.comb_batch(batch.a_blob, batch.b_blob, batch.a_off, batch.b_off, batch.ms, batch.ns, off, total)


@pytest.mark.parametrize("graph,tns,bpsm", [(0, 8, 0), (1, 8, 0), (0, 4, 0), (1, 8, 1), (0, 4, 2)])
def test_batch_reads(cuda, graph, tns, bpsm):
    """Default stream plan: every pair in the smallest row class (32-bit
    strands), or, with 4 columns per step, the variable packed class whose
    segments take any lane count."""
    import torch
    batch = W.reads_20000(npairs=3000)
    descs = slcs.pair_descs(batch)
    _, total = batch.strand_offsets()
    out = torch.empty(total, dtype=torch.int32, device=cuda)
    plan = slcs.BatchPlan(descs, slcs.Config.make(use_graph=graph, tile_n=tns, blocks_per_sm=bpsm))
    assert plan.info["stream_classes"] >= (1 if tns == 4 else 3) and plan.info["tile_n"] == tns
    a_d, b_d = _dev(batch.a_blob, cuda), _dev(batch.b_blob, cuda)
    want = _batch_expected(batch)
    for _ in range(2):
        out.fill_(-7)
        plan.run(a_d, b_d, out)
        torch.cuda.synchronize()
        slcs.device_status(0)
        np.testing.assert_array_equal(out.cpu().numpy(), want)


def _mixed_batch(seed, count=300, mmax=1500, nmax=1500):
    rng = np.random.default_rng(seed)
    pairs = []
    for _ in range(count):
        m = int(rng.integers(0, mmax)); n = int(rng.integers(0, nmax))
        sigma = int(rng.choice([2, 4, 256]))
        pairs.append((rng.integers(0, sigma, m, dtype=np.uint8), rng.integers(0, sigma, n, dtype=np.uint8)))
    return W.pack(pairs)


def test_batch_mixed_sizes_wavefront(cuda):
    import torch
    batch = _mixed_batch(11)
    descs = slcs.pair_descs(batch)
    _, total = batch.strand_offsets()
    want = _batch_expected(batch)
    for tm in (2, 8, 16):
        out = torch.full((total,), -7, dtype=torch.int32, device=cuda)
        slcs.comb_batch(descs, _dev(batch.a_blob, cuda), _dev(batch.b_blob, cuda), out,
                        slcs.Config.make(algo=slcs.ALGO_WAVEFRONT, tile_m=tm))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), want)
    host = slcs.comb_batch_host(descs, batch.a_blob, batch.b_blob, total)
    np.testing.assert_array_equal(host, want)


@pytest.mark.parametrize("stm,seg,tns", [(4, 8, 4), (4, 32, 8), (8, 16, 4), (12, 16, 8), (16, 8, 8), (16, 16, 4),
                                         (16, 32, 8)])
def test_batch_stream_variants(cuda, stm, seg, tns):
    """Stream mode (pairs of at most seg*stm rows) plus wavefront tasks for the rest."""
    import torch
    batch = _mixed_batch(20 + stm + seg, count=400, mmax=700, nmax=900)
    descs = slcs.pair_descs(batch)
    _, total = batch.strand_offsets()
    want = _batch_expected(batch)
    plan = slcs.BatchPlan(descs, slcs.Config.make(tile_m=stm, seg=seg, tile_n=tns))
    info = plan.info
    assert info["stream_tile_m"] == stm and info["seg"] == seg and info["stream_pairs"] > 0
    out = torch.full((total,), -7, dtype=torch.int32, device=cuda)
    plan.run(_dev(batch.a_blob, cuda), _dev(batch.b_blob, cuda), out)
    torch.cuda.synchronize()
    slcs.device_status(0)
    np.testing.assert_array_equal(out.cpu().numpy(), want)


def test_batch_stream_tiny_pairs(cuda):
    """Pairs of one block or less: the segment switches pairs every step."""
    import torch
    rng = np.random.default_rng(99)
    pairs = [(rng.integers(0, 3, int(rng.integers(1, 9)), dtype=np.uint8),
              rng.integers(0, 3, int(rng.integers(1, 6)), dtype=np.uint8)) for _ in range(500)]
    batch = W.pack(pairs)
    descs = slcs.pair_descs(batch)
    _, total = batch.strand_offsets()
    for seg in (8, 16, 32):
        out = torch.full((total,), -7, dtype=torch.int32, device=cuda)
        plan = slcs.BatchPlan(descs, slcs.Config.make(tile_m=4, seg=seg))
        plan.run(_dev(batch.a_blob, cuda), _dev(batch.b_blob, cuda), out)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), _batch_expected(batch))


def _pack_unaligned(pairs, seed):
    """Like workloads.pack, but every string starts at a random byte offset."""
    rng = np.random.default_rng(seed)

    def blob(strings):
        off = np.zeros(len(strings), np.int64)
        pos = 0
        for i, s in enumerate(strings):
            pos += int(rng.integers(0, 4))
            off[i] = pos
            pos += len(s)
        buf = np.zeros(pos + 16, np.uint8)
        for o, s in zip(off, strings):
            buf[o:o + len(s)] = s
        return buf, off

    a_blob, a_off = blob([a for a, _ in pairs])
    b_blob, b_off = blob([b for _, b in pairs])
    return W.Batch(a_blob, b_blob, a_off, b_off, np.array([len(a) for a, _ in pairs], np.int32),
                   np.array([len(b) for _, b in pairs], np.int32))


def _run_plan(batch, cfg, cuda):
    import torch
    descs = slcs.pair_descs(batch)
    _, total = batch.strand_offsets()
    plan = slcs.BatchPlan(descs, cfg)
    out = torch.full((total,), -7, dtype=torch.int32, device=cuda)
    plan.run(_dev(batch.a_blob, cuda), _dev(batch.b_blob, cuda), out)
    torch.cuda.synchronize()
    slcs.device_status(0)
    info = plan.info
    plan.close()
    return out.cpu().numpy(), info


def test_batch_packed_reads_match_32bit(cuda):
    """Default plan on read pairs combs two pairs per register; forcing 32-bit
    strands gives the same strands."""
    batch = W.reads_20000(npairs=2001)
    want = _batch_expected(batch)
    got, info = _run_plan(batch, slcs.Config.make(), cuda)
    assert info["packed_pairs"] > 1000 and info["tile_n"] == 4
    np.testing.assert_array_equal(got, want)
    got32, info32 = _run_plan(batch, slcs.Config.make(strand_bits=32), cuda)
    assert info32["packed_pairs"] == 0
    np.testing.assert_array_equal(got32, want)


def _packed_class_pairs(stm):
    rng = np.random.default_rng(300 + stm)
    rows = 16 * stm
    pairs = []
    for i in range(161):
        m = int(rng.integers(1, rows + 1))
        n = int(rng.integers(1, 700))
        if i % 40 == 0:
            n = 32767 - m
        elif i % 40 == 1:
            n = 32768 - m
        elif i % 53 == 5:
            n = 0
        sigma = int(rng.choice([2, 4, 20, 256]))
        pairs.append((rng.integers(0, sigma, m, dtype=np.uint8), rng.integers(0, sigma, n, dtype=np.uint8)))
    return pairs


@pytest.mark.parametrize("stm", [4, 8, 12, 16])
def test_batch_packed_classes(cuda, stm):
    """One packed class plus its 32-bit twin: an odd pair count, pairs whose
    ids just fit 15 bits (m + n = 32767) and pairs just past it (32768, not
    packable), unaligned strings, shorter partners, empty sides."""
    pairs = _packed_class_pairs(stm)
    batch = _pack_unaligned(pairs, stm)
    want = _batch_expected(batch)
    got, info = _run_plan(batch, slcs.Config.make(tile_m=stm, seg=16, tile_n=4), cuda)
    eligible = sum(1 for a, b in pairs if len(b) > 0 and len(a) + len(b) <= 32767)
    assert info["packed_pairs"] == eligible
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("tns", [4, 8])
def test_batch_stream_unaligned_strings(cuda, tns):
    """32-bit stream classes on strings at odd byte offsets."""
    pairs = _packed_class_pairs(16)
    batch = _pack_unaligned(pairs, 5 + tns)
    got, info = _run_plan(batch, slcs.Config.make(strand_bits=32, tile_n=tns), cuda)
    assert info["packed_pairs"] == 0 and info["stream_pairs"] > 100
    np.testing.assert_array_equal(got, _batch_expected(batch))


def test_batch_packed_tiny_pairs(cuda):
    """Couples of one-block pairs switch every step."""
    rng = np.random.default_rng(77)
    pairs = [(rng.integers(0, 3, int(rng.integers(1, 40)), dtype=np.uint8),
              rng.integers(0, 3, int(rng.integers(1, 9)), dtype=np.uint8)) for _ in range(777)]
    batch = W.pack(pairs)
    got, info = _run_plan(batch, slcs.Config.make(tile_n=4), cuda)
    assert info["packed_pairs"] == 777
    np.testing.assert_array_equal(got, _batch_expected(batch))


def _golden():
    import json
    import os
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.json")) as f:
        return json.load(f)


def _sha256(x):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(x).tobytes()).hexdigest()


@pytest.mark.parametrize("name,cfg", [("pair_131072_mutated", dict()),
                                      ("pair_1M", dict(tile_m=16, warps=8)),
                                      ("pair_1M", dict())])
def test_pair_large_golden(cuda, name, cfg):
    """Full-size single pairs against digests of the oracle's permutation
    (tests/golden/make_golden.py --big wrote them)."""
    g = _golden()[name]
    a, b = W.pair_131072_mutated() if name == "pair_131072_mutated" else W.pair_1m()
    h, v = slcs.comb_pair(_dev(a, cuda), _dev(b, cuda), cfg=slcs.Config.make(**cfg))
    _, c2r = slcs.strands_to_permutation(h, v)
    c2r = c2r.cpu().numpy()
    slcs.device_status(0)
    assert _sha256(c2r) == g["sha256_col_to_row"]
    assert slcs.permutation_hash(c2r) == g["hash"]


@pytest.mark.parametrize("cfg", [dict(), dict(strand_bits=32), dict(tile_n=8), dict(algo=1, tile_m=8)])
def test_batch_reads_20000_golden(cuda, cfg):
    """The 20,000-read batch against the digest of the oracle's strands."""
    g = _golden()["reads_20000"]
    batch = W.reads_20000()
    assert batch.cells == g["cells"]
    got, _ = _run_plan(batch, slcs.Config.make(**cfg), cuda)
    assert _sha256(got) == g["sha256_strands"]


def test_batch_default_plan_all_row_classes(cuda):
    """Rows 1..600 through the default plan: the variable packed class
    (segments of 4..32 lanes sharing warps, idle lanes where they do not fill
    one), 32-bit classes for the pairs whose ids need more than 15 bits, and
    wavefront tasks for pairs taller than 512 rows."""
    rng = np.random.default_rng(4242)
    pairs = []
    for i in range(1201):
        m = int(rng.integers(1, 601))
        n = int(rng.integers(1, 400)) if i % 97 else 32768 - min(m, 256)  # not packable
        sigma = int(rng.choice([2, 4, 256]))
        pairs.append((rng.integers(0, sigma, m, dtype=np.uint8), rng.integers(0, sigma, n, dtype=np.uint8)))
    batch = _pack_unaligned(pairs, 4242)
    got, info = _run_plan(batch, slcs.Config.make(), cuda)
    assert info["stream_classes"] >= 2 and info["packed_pairs"] > 0 and info["wavefront_tasks"] > 0
    np.testing.assert_array_equal(got, _batch_expected(batch))


@pytest.mark.parametrize("pinned", [True, False])
def test_batch_run_host_chunked_golden(cuda, pinned):
    """Host run of the 20,000-read batch (cut into chunks whose copies overlap
    the combing of other chunks) against the oracle's digest, twice."""
    import torch
    g = _golden()["reads_20000"]
    batch = W.reads_20000()
    descs = slcs.pair_descs(batch)
    _, total = batch.strand_offsets()
    plan = slcs.BatchPlan(descs, slcs.Config.make(use_graph=1))
    if pinned:
        a = torch.from_numpy(batch.a_blob).pin_memory().numpy()
        b = torch.from_numpy(batch.b_blob).pin_memory().numpy()
        out = torch.empty(total, dtype=torch.int32).pin_memory().numpy()
    else:
        a, b, out = batch.a_blob, batch.b_blob, np.empty(total, np.int32)
    for _ in range(2):
        out[:] = -7
        plan.run_host(a, b, out)
        assert _sha256(out) == g["sha256_strands"]
    plan.close()


def test_batch_run_host_chunked_ragged(cuda):
    """More than 8192 pairs with empty sides and odd offsets through the host
    run, against the oracle."""
    rng = np.random.default_rng(515)
    pairs = []
    for i in range(9001):
        m = int(rng.integers(0, 300)) if i % 37 else 0
        n = int(rng.integers(0, 400)) if i % 41 else 0
        pairs.append((rng.integers(0, 4, m, dtype=np.uint8), rng.integers(0, 4, n, dtype=np.uint8)))
    batch = _pack_unaligned(pairs, 515)
    descs = slcs.pair_descs(batch)
    _, total = batch.strand_offsets()
    plan = slcs.BatchPlan(descs, slcs.Config.make())
    out = np.full(total, -7, np.int32)
    plan.run_host(batch.a_blob, batch.b_blob, out)
    np.testing.assert_array_equal(out, _batch_expected(batch))
    plan.close()


def test_batch_host_run_int16_strands(cuda):
    """slcs_batch_plan_run_host16 returns the int32 run's strands as int16,
    through the chunked path (20,000 reads) and the single-launch path (a
    small batch); a plan with a pair of m + n > 32767 is refused."""
    for batch in (W.reads_20000(), W.reads_20000(npairs=300, seed=9)):
        _, total = batch.strand_offsets()
        plan = slcs.BatchPlan(slcs.pair_descs(batch))
        o32 = np.empty(total, np.int32)
        o16 = np.full(total, -7, np.int16)
        plan.run_host(batch.a_blob, batch.b_blob, o32)
        plan.run_host16(batch.a_blob, batch.b_blob, o16)
        assert np.array_equal(o16.astype(np.int32), o32)
        plan.close()
    big = W.pack([(np.zeros(20000, np.uint8), np.zeros(13000, np.uint8))])
    plan = slcs.BatchPlan(slcs.pair_descs(big))
    with pytest.raises(slcs.SlcsError) as err:
        plan.run_host16(big.a_blob, big.b_blob, np.empty(33000, np.int16))
    assert err.value.status == 6
    plan.close()
