"""Failure detection on the device, in the form that leaves the GPU usable: a
bounded wait that nothing satisfies runs out, the launch ends, and the host
reads an error status (the reference reports failures by exceptions caught in
src/main.cpp:83-94).  Nothing here faults, traps or hangs a GPU."""
import time

import numpy as np
import pytest

import oracle as O
import slcs

pytestmark = pytest.mark.gpu


def test_bounded_wait_expiry_reports_timeout_and_context_survives(cuda):
    import torch
    torch.cuda.synchronize()
    slcs.device_status(0)  # start from a clear status word
    t0 = time.perf_counter()
    slcs.probe_wait_expiry(200)
    torch.cuda.synchronize()
    waited = time.perf_counter() - t0
    with pytest.raises(slcs.SlcsError) as err:
        slcs.device_status(0)
    assert err.value.status == 4  # SLCS_ERR_TIMEOUT
    assert 0.15 <= waited < 5.0
    slcs.device_status(0)  # the error was cleared by the read above
    # the next call on the same context runs normally and bit-exactly
    rng = np.random.default_rng(17)
    a = rng.integers(0, 4, 700, dtype=np.uint8)
    b = rng.integers(0, 4, 333, dtype=np.uint8)
    h, v = slcs.comb_pair(torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda),
                          cfg=slcs.Config.make(tile_m=2))
    torch.cuda.synchronize()
    slcs.device_status(0)
    eh, ev = O.comb(a, b)
    assert np.array_equal(h.cpu().numpy(), eh) and np.array_equal(v.cpu().numpy(), ev)


def test_wait_expiry_argument_range(cuda):
    with pytest.raises(slcs.SlcsError) as err:
        slcs.probe_wait_expiry(0)
    assert err.value.status == 6
