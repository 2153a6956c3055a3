"""ctypes front end of the CPU oracle.

TEST INFRASTRUCTURE ONLY: tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this
module, and only as the checker or as the timed CPU baseline.  The product
path (``slcs``) never imports it.

Two libraries sit behind it:

* ``_build/liboracle.so`` -- the plain-C restatement in ``slcs_oracle.c``.
* ``_ref/libslcs_ref.so`` -- the reference's own CPU code (``src/lcs_residual_fixup.hpp``,
  ``src/permutation_matrix.hpp``, ``src/braid_multiplication.hpp``) compiled in
  place by ``oracle/Makefile``.  It is optional at run time; tests that need it
  skip when it is absent.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def _ptr(arr, ty):
    return arr.ctypes.data_as(ty)


def build(ref_src: str | None = None):
    """Compile the oracle; with ``ref_src`` (the reference's ``src/``
    directory, else the ``SLCS_REF_SRC`` environment variable) also the
    reference bridge."""
    ref_src = ref_src or os.environ.get("SLCS_REF_SRC")
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if ref_src:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF_SRC={ref_src}"], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "_build", "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.oracle_comb_u8.argtypes = [_u8p, ctypes.c_int32, _u8p, ctypes.c_int32, _i32p, _i32p]
        L.oracle_comb_i32.argtypes = [_i32p, ctypes.c_int32, _i32p, ctypes.c_int32, _i32p, _i32p]
        L.oracle_comb_batch_u8.argtypes = [ctypes.c_int32, _i64p, _i64p, _i32p, _i32p, _u8p, _u8p,
                                           _i64p, _i32p, ctypes.c_int32]
        L.oracle_from_strands.argtypes = [_i32p, ctypes.c_int32, _i32p, ctypes.c_int32, _i32p, _i32p]
        L.oracle_hash.argtypes = [_i32p, ctypes.c_int32]
        L.oracle_hash.restype = ctypes.c_int64
        L.oracle_staggered_multiply.argtypes = [_i32p, ctypes.c_int32, _i32p, ctypes.c_int32,
                                                ctypes.c_int32, ctypes.c_int32, _i32p, _i32p]
        L.oracle_staggered_multiply.restype = ctypes.c_int32
        L.oracle_llcs_from_strands.argtypes = [_i32p, ctypes.c_int32, _i32p, ctypes.c_int32]
        L.oracle_llcs_from_strands.restype = ctypes.c_int32
        L.oracle_prefix_llcs_u8.argtypes = [_u8p, ctypes.c_int32, _u8p, ctypes.c_int32]
        L.oracle_prefix_llcs_u8.restype = ctypes.c_int32
        L.oracle_comb_strips_u8.argtypes = [_u8p, ctypes.c_int32, _u8p, ctypes.c_int32, ctypes.c_int32,
                                            ctypes.c_int32, _i32p]
        L.oracle_comb_strips_u8.restype = ctypes.c_int32
        _LIB = L
    return _LIB


def ref_lib():
    """The reference's own code, or None when oracle/_ref was never built."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libslcs_ref.so")
        if not os.path.exists(path):
            if os.environ.get("SLCS_REF_SRC"):
                build()
            if not os.path.exists(path):
                return None
        L = ctypes.CDLL(path)
        L.ref_comb_i32.argtypes = [_i32p, ctypes.c_int32, _i32p, ctypes.c_int32, _i32p, _i32p]
        L.ref_comb_batch_i32.argtypes = [ctypes.c_int32, _i64p, _i64p, _i32p, _i32p, _i32p, _i32p,
                                         _i64p, _i32p, ctypes.c_int32]
        L.ref_hash_from_strands.argtypes = [_i32p, ctypes.c_int32, _i32p, ctypes.c_int32, _i32p]
        L.ref_hash_from_strands.restype = ctypes.c_int64
        L.ref_hash_col_to_row.argtypes = [_i32p, ctypes.c_int32]
        L.ref_hash_col_to_row.restype = ctypes.c_int64
        L.ref_staggered_multiply.argtypes = [_i32p, ctypes.c_int32, _i32p, ctypes.c_int32,
                                             ctypes.c_int32, ctypes.c_int32, _i32p, _i32p]
        L.ref_comb_strips_i32.argtypes = [_i32p, ctypes.c_int32, _i32p, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_int32, _i32p]
        _REF = L
    return _REF


# --------------------------------------------------------------------------
# oracle wrappers (numpy in, numpy out)
# --------------------------------------------------------------------------

def comb(a: np.ndarray, b: np.ndarray):
    """(h, v) strands of one pair of uint8 strings."""
    a = np.ascontiguousarray(a, dtype=np.uint8)
    b = np.ascontiguousarray(b, dtype=np.uint8)
    h = np.empty(len(a), np.int32)
    v = np.empty(len(b), np.int32)
    lib().oracle_comb_u8(_ptr(a, _u8p), len(a), _ptr(b, _u8p), len(b), _ptr(h, _i32p), _ptr(v, _i32p))
    return h, v


def comb_antidiagonal(a: np.ndarray, b: np.ndarray):
    """Same as comb() with the reference's literal anti-diagonal visiting order."""
    a = np.ascontiguousarray(a, dtype=np.int32)
    b = np.ascontiguousarray(b, dtype=np.int32)
    h = np.empty(len(a), np.int32)
    v = np.empty(len(b), np.int32)
    lib().oracle_comb_i32(_ptr(a, _i32p), len(a), _ptr(b, _i32p), len(b), _ptr(h, _i32p), _ptr(v, _i32p))
    return h, v


def comb_batch(a_blob, b_blob, a_off, b_off, ms, ns, out_off, out_len, nthreads=None):
    """Strands of many pairs; the output blob holds h then v of each pair."""
    nthreads = nthreads or os.cpu_count() or 1
    out = np.zeros(out_len, np.int32)
    a_off = np.ascontiguousarray(a_off, np.int64)
    b_off = np.ascontiguousarray(b_off, np.int64)
    out_off = np.ascontiguousarray(out_off, np.int64)
    ms = np.ascontiguousarray(ms, np.int32)
    ns = np.ascontiguousarray(ns, np.int32)
    a_blob = np.ascontiguousarray(a_blob, np.uint8)
    b_blob = np.ascontiguousarray(b_blob, np.uint8)
    lib().oracle_comb_batch_u8(len(ms), _ptr(a_off, _i64p), _ptr(b_off, _i64p), _ptr(ms, _i32p),
                               _ptr(ns, _i32p), _ptr(a_blob, _u8p), _ptr(b_blob, _u8p),
                               _ptr(out_off, _i64p), _ptr(out, _i32p), int(nthreads))
    return out


def from_strands(h, v):
    """(row_to_col, col_to_row) of PermutationMatrix::FromStrands."""
    h = np.ascontiguousarray(h, np.int32)
    v = np.ascontiguousarray(v, np.int32)
    size = len(h) + len(v)
    r2c = np.empty(size, np.int32)
    c2r = np.empty(size, np.int32)
    lib().oracle_from_strands(_ptr(h, _i32p), len(h), _ptr(v, _i32p), len(v), _ptr(r2c, _i32p), _ptr(c2r, _i32p))
    return r2c, c2r


def perm_hash(col_to_row) -> int:
    c = np.ascontiguousarray(col_to_row, np.int32)
    return int(lib().oracle_hash(_ptr(c, _i32p), len(c)))


def staggered_multiply(p_r2c, q_r2c, k: int, row_glue: bool):
    p = np.ascontiguousarray(p_r2c, np.int32)
    q = np.ascontiguousarray(q_r2c, np.int32)
    size = len(p) + len(q) - k
    r2c = np.empty(size, np.int32)
    c2r = np.empty(size, np.int32)
    rc = lib().oracle_staggered_multiply(_ptr(p, _i32p), len(p), _ptr(q, _i32p), len(q), k, int(row_glue),
                                         _ptr(r2c, _i32p), _ptr(c2r, _i32p))
    if rc != 0:
        raise ValueError("oracle_staggered_multiply: bad arguments")
    return r2c, c2r


def llcs_from_strands(h, v) -> int:
    h = np.ascontiguousarray(h, np.int32)
    v = np.ascontiguousarray(v, np.int32)
    return int(lib().oracle_llcs_from_strands(_ptr(h, _i32p), len(h), _ptr(v, _i32p), len(v)))


def prefix_llcs(a, b) -> int:
    a = np.ascontiguousarray(a, np.uint8)
    b = np.ascontiguousarray(b, np.uint8)
    return int(lib().oracle_prefix_llcs_u8(_ptr(a, _u8p), len(a), _ptr(b, _u8p), len(b)))


def comb_strips(a, b, strips: int, nthreads=None):
    """col_to_row of one large pair by strip combing plus a staggered-multiply tree."""
    nthreads = nthreads or os.cpu_count() or 1
    a = np.ascontiguousarray(a, np.uint8)
    b = np.ascontiguousarray(b, np.uint8)
    c2r = np.empty(len(a) + len(b), np.int32)
    lib().oracle_comb_strips_u8(_ptr(a, _u8p), len(a), _ptr(b, _u8p), len(b), int(strips), int(nthreads),
                                _ptr(c2r, _i32p))
    return c2r


def comb_tiles(a, b, heights, widths):
    """row_to_col of P(a, b) from tiles: a cut into row bands of the given
    heights, b into column strips of the given widths; every tile combed
    apart, each band's strips glued left to right by
    staggered_multiply<false> with overlap = band height, then the bands top
    to bottom by staggered_multiply<true> with overlap = len(b)
    (src/braid_multiplication.hpp:273-407).  The library's tile mode merges
    in this order (balanced trees instead of left to right chains)."""
    a = np.ascontiguousarray(a, np.uint8)
    b = np.ascontiguousarray(b, np.uint8)
    assert sum(heights) == len(a) and sum(widths) == len(b)
    band_perms = []
    r0 = 0
    for hgt in heights:
        c0 = 0
        P = None
        for w in widths:
            T = from_strands(*comb(a[r0:r0 + hgt], b[c0:c0 + w]))[0]
            P = T if P is None else staggered_multiply(P, T, hgt, False)[0]
            c0 += w
        band_perms.append(P)
        r0 += hgt
    P = band_perms[0]
    for Q in band_perms[1:]:
        P = staggered_multiply(P, Q, len(b), True)[0]
    return P


# --------------------------------------------------------------------------
# reference wrappers
# --------------------------------------------------------------------------

def ref_comb(a, b):
    L = ref_lib()
    a = np.ascontiguousarray(a, np.int32)
    b = np.ascontiguousarray(b, np.int32)
    h = np.empty(len(a), np.int32)
    v = np.empty(len(b), np.int32)
    L.ref_comb_i32(_ptr(a, _i32p), len(a), _ptr(b, _i32p), len(b), _ptr(h, _i32p), _ptr(v, _i32p))
    return h, v


def ref_hash_from_strands(h, v):
    L = ref_lib()
    h = np.ascontiguousarray(h, np.int32)
    v = np.ascontiguousarray(v, np.int32)
    c2r = np.empty(len(h) + len(v), np.int32)
    hv = L.ref_hash_from_strands(_ptr(h, _i32p), len(h), _ptr(v, _i32p), len(v), _ptr(c2r, _i32p))
    return int(hv), c2r


def ref_staggered_multiply(p_r2c, q_r2c, k: int, row_glue: bool):
    L = ref_lib()
    p = np.ascontiguousarray(p_r2c, np.int32)
    q = np.ascontiguousarray(q_r2c, np.int32)
    size = len(p) + len(q) - k
    r2c = np.empty(size, np.int32)
    c2r = np.empty(size, np.int32)
    L.ref_staggered_multiply(_ptr(p, _i32p), len(p), _ptr(q, _i32p), len(q), k, int(row_glue),
                             _ptr(r2c, _i32p), _ptr(c2r, _i32p))
    return r2c, c2r


def ref_comb_batch(a_blob_i32, b_blob_i32, a_off, b_off, ms, ns, out_off, out_len, nthreads=None):
    L = ref_lib()
    nthreads = nthreads or os.cpu_count() or 1
    out = np.zeros(out_len, np.int32)
    args = [np.ascontiguousarray(x, t) for x, t in ((a_off, np.int64), (b_off, np.int64), (ms, np.int32),
                                                    (ns, np.int32), (a_blob_i32, np.int32),
                                                    (b_blob_i32, np.int32), (out_off, np.int64))]
    a_off, b_off, ms, ns, ab, bb, out_off = args
    L.ref_comb_batch_i32(len(ms), _ptr(a_off, _i64p), _ptr(b_off, _i64p), _ptr(ms, _i32p), _ptr(ns, _i32p),
                         _ptr(ab, _i32p), _ptr(bb, _i32p), _ptr(out_off, _i64p), _ptr(out, _i32p), int(nthreads))
    return out


def ref_comb_strips(a, b, strips: int, nthreads=None):
    """col_to_row of one large pair from reference functions only (strips + merges)."""
    L = ref_lib()
    nthreads = nthreads or os.cpu_count() or 1
    a = np.ascontiguousarray(a, np.int32)
    b = np.ascontiguousarray(b, np.int32)
    c2r = np.empty(len(a) + len(b), np.int32)
    L.ref_comb_strips_i32(_ptr(a, _i32p), len(a), _ptr(b, _i32p), len(b), int(strips), int(nthreads),
                          _ptr(c2r, _i32p))
    return c2r


def mt19937_binary(size: int, seed: int) -> np.ndarray:
    """generate_random_binary_sequence (src/test_utility.hpp:8-18): std::mt19937
    seeded with `seed`, one draw per symbol, keep the lowest bit.  numpy's legacy
    RandomState seeding is the same init_genrand routine as std::mt19937."""
    bg = np.random.RandomState(seed)._bit_generator
    raw = bg.random_raw(size)
    return (raw & 1).astype(np.uint8)


def substring_llcs(v, m: int, begin, end):
    """LLCS(a, b[i, j)) = (j - i) - #{k in [i, j) : v[k] >= m + i} from the
    v strands of the comb of (a, b) (the semi-local string-substring solution;
    checked against the DP of prefix_llcs in the tests)."""
    v = np.asarray(v)
    out = np.empty(len(begin), np.int64)
    for q, (i, j) in enumerate(zip(begin, end)):
        out[q] = (j - i) - int(np.count_nonzero(v[i:j] >= m + i))
    return out
