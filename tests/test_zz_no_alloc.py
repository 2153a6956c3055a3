"""slcs_comb_pair_noalloc: the entry point for callers that cannot allocate
device memory when they call (for example while a stream is being captured
into a CUDA graph with allocation disallowed, or in a service that reserved
all device memory up front).  Its scratch lives in one fixed device array;
its strands must equal those of the allocating slcs_comb_pair.

This file is collected last on purpose; it also passes alone in a fresh
process, where its first call is the one that looks up the array."""
import ctypes

import numpy as np
import pytest

import slcs

pytestmark = pytest.mark.gpu

_vp = ctypes.c_void_p
_i32 = ctypes.c_int32


def _entry():
    L = slcs.lib()
    f = L.slcs_comb_pair_noalloc
    f.argtypes = [_vp, _i32, _vp, _i32, _vp, ctypes.POINTER(slcs.Config), _vp]
    f.restype = _i32
    return f


def _pair(seed, m, n, sigma=4):
    rng = np.random.default_rng(seed)
    return rng.integers(0, sigma, m, dtype=np.uint8), rng.integers(0, sigma, n, dtype=np.uint8)


# (seed, m, n, tile_m): multi-stripe shapes (many rows per pair), so the fixed
# scratch carries the strands between stripes.  (5, 160000, 300, 2) has 2500
# stripes, more than 16 warps on every SM of a B200, so its launch is the
# persistent one that takes stripes from the ticket counter; (6, 600000, 211,
# None) takes the tall-pair rule (14 or 16 rows per lane), which
# slcs_comb_pair combs as row bands glued by braid products instead.
SHAPES = [(1, 3001, 2503, 2), (2, 4096, 777, 4), (3, 1000, 4097, 8), (4, 37, 5, 2), (5, 160000, 300, 2),
          (6, 600000, 211, None)]


def test_noalloc_matches_allocating_entry(cuda):
    import torch
    f = _entry()
    stream = torch.cuda.current_stream().cuda_stream
    for seed, m, n, tm in SHAPES:
        a, b = _pair(seed, m, n)
        ad = torch.from_numpy(a).to(cuda)
        bd = torch.from_numpy(b).to(cuda)
        cfg = slcs.Config.make(tile_m=tm)
        want = torch.empty(m + n, dtype=torch.int32, device=cuda)
        slcs.comb_pair(ad, bd, cfg=cfg, out=want)
        # two calls in a row: the second finds the array as the first left it
        for _ in range(2):
            got = torch.full((m + n,), -7, dtype=torch.int32, device=cuda)
            rc = f(ad.data_ptr(), m, bd.data_ptr(), n, got.data_ptr(), ctypes.byref(cfg), stream)
            assert rc == 0, slcs.lib().slcs_last_error()
            torch.cuda.synchronize()
            slcs.device_status(0)
            assert torch.equal(got, want), (seed, m, n)


def test_noalloc_empty_side_and_limit(cuda):
    import torch
    f = _entry()
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.full((9,), -7, dtype=torch.int32, device=cuda)
    a = torch.zeros(9, dtype=torch.uint8, device=cuda)
    assert f(a.data_ptr(), 9, None, 0, out.data_ptr(), None, stream) == 0
    torch.cuda.synchronize()
    assert out.cpu().tolist() == list(range(9))
    # A pair whose hand-down row would not fit the fixed array is refused from
    # its sizes alone, before any pointer is looked at: with null pointers a
    # refusal that went missing would end in SLCS_ERR_INVALID, never on the GPU.
    limit = 16 << 20
    cfg = slcs.Config.make(tile_m=2)
    assert f(None, 65, None, limit // 4 + 64, None, ctypes.byref(cfg), stream) == 6
    assert b"SLCS_NOALLOC_SCRATCH_BYTES" in slcs.lib().slcs_last_error()
