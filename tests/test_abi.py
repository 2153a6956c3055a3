"""The C ABI library loads and exports every symbol include/slcs.h declares;
host-only entry points and argument checks work without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle as O
import slcs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(macro="SLCS_API"):
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(macro + r"[^;{(]*?\b(slcs_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    L = slcs.lib()
    names = _declared()
    assert len(names) >= 15
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_host_library_exports_its_c_entry_points():
    H = slcs.host_lib()
    names = _declared("SLCS_HOST_API")
    assert "slcs_host_run_procedure" in names
    missing = [n for n in sorted(names) if not hasattr(H, n)]
    assert not missing, missing


def test_struct_layouts():
    assert ctypes.sizeof(slcs.Config) == 16 * 4
    assert ctypes.sizeof(slcs.PairDesc) == 32
    assert slcs.PAIR_DTYPE.itemsize == 32


def test_status_strings():
    L = slcs.lib()
    assert L.slcs_status_string(0) == b"ok"
    assert L.slcs_status_string(4) == b"device wait timed out"
    assert L.slcs_version() >= 1


def test_host_hash_matches_reference_definition():
    rng = np.random.default_rng(0)
    for size in (1, 2, 17, 1000, 8192):
        c2r = rng.permutation(size).astype(np.int32)
        assert slcs.permutation_hash(c2r) == O.perm_hash(c2r)
    a, b = O.mt19937_binary(7330, 888), O.mt19937_binary(9944, 999)
    assert slcs.permutation_hash(O.from_strands(*O.comb(a, b))[1]) == 944438867


def test_argument_checks_fail_before_touching_the_device():
    L = slcs.lib()
    assert L.slcs_comb_pair(None, -1, None, 3, None, None, None, None) == 1
    assert L.slcs_comb_pair(None, 3, None, 3, None, None, None, None) == 1
    assert b"null" in L.slcs_last_error()
    assert L.slcs_comb_pair_host(None, 5, None, 0, None, None, None) == 1
    bad = np.zeros(1, slcs.PAIR_DTYPE)
    bad["m"] = -4
    assert L.slcs_comb_batch_host(bad.ctypes.data, 1, None, 0, None, 0, None, 0, None) == 1
    big = np.zeros(1, slcs.PAIR_DTYPE)
    big["m"], big["n"] = 2**31 - 10, 100
    assert L.slcs_batch_plan_create(ctypes.byref(ctypes.c_void_p()), big.ctypes.data, 1, None) == 6
    with pytest.raises(slcs.SlcsError):
        slcs.check(1)


def test_noalloc_refuses_oversized_scratch_without_a_device():
    """The allocation-free entry point refuses a pair whose scratch exceeds its
    fixed array from the sizes alone (null pointers, no device needed)."""
    L = slcs.lib()
    f = L.slcs_comb_pair_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                  ctypes.POINTER(slcs.Config), ctypes.c_void_p]
    cfg = slcs.Config.make(tile_m=2)
    assert f(None, 65, None, (16 << 20) // 4 + 64, None, ctypes.byref(cfg), None) == 6
    assert b"SLCS_NOALLOC_SCRATCH_BYTES" in L.slcs_last_error()
    assert f(None, 65, None, 1000, None, ctypes.byref(cfg), None) == 1  # fits: then the null pointers


def test_host_adapter_unknown_procedure_without_a_device():
    """An unknown name is the reference's impl.ok == false: reported before any
    device work."""
    rc, _, _, _, _, msg = slcs.run_procedure("no_such_procedure", np.zeros(3, np.int32), np.zeros(2, np.int32))
    assert rc == 1 and "no_such_procedure" in msg
