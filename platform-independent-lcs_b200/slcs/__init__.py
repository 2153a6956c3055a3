"""Python binding of libslcs.so (the B200 semi-local LCS engine).

The binding is a thin ctypes layer over the C ABI declared in include/slcs.h.
There is no CPU fallback: if the CUDA library is missing, every entry point
raises.  Device buffers are torch CUDA tensors (torch is used for device
memory and streams only); host buffers are numpy arrays.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT_DIR = os.path.dirname(PKG_DIR)
LIB_PATH = os.path.join(ROOT_DIR, "lib", "libslcs.so")
HOST_LIB_PATH = os.path.join(ROOT_DIR, "lib", "libslcs_host.so")

ALGO_AUTO, ALGO_WAVEFRONT, ALGO_STRIPS = 0, 1, 2


class SlcsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"slcs status {status}: {message}")
        self.status = status


class Config(ctypes.Structure):
    _fields_ = [("algo", ctypes.c_int32), ("tile_m", ctypes.c_int32), ("tile_n", ctypes.c_int32),
                ("warps", ctypes.c_int32), ("braid_cutoff", ctypes.c_int32), ("strips", ctypes.c_int32),
                ("use_graph", ctypes.c_int32), ("seg", ctypes.c_int32), ("wait_ms", ctypes.c_int32),
                ("blocks_per_sm", ctypes.c_int32), ("strand_bits", ctypes.c_int32), ("bands", ctypes.c_int32),
                ("pool_pct", ctypes.c_int32), ("reserved", ctypes.c_int32 * 3)]

    @classmethod
    def make(cls, **kw) -> "Config":
        c = cls()
        for k, v in kw.items():
            if v is not None:
                setattr(c, k, int(v))
        return c


class PairDesc(ctypes.Structure):
    _fields_ = [("a_offset", ctypes.c_int64), ("b_offset", ctypes.c_int64), ("out_offset", ctypes.c_int64),
                ("m", ctypes.c_int32), ("n", ctypes.c_int32)]


class PlanInfo(ctypes.Structure):
    _fields_ = [("stream_tile_m", ctypes.c_int32), ("seg", ctypes.c_int32), ("wavefront_tile_m", ctypes.c_int32),
                ("warps", ctypes.c_int32), ("stream_pairs", ctypes.c_int32), ("wavefront_tasks", ctypes.c_int32),
                ("stream_classes", ctypes.c_int32), ("tile_n", ctypes.c_int32), ("grid", ctypes.c_int32),
                ("packed_pairs", ctypes.c_int32), ("reserved", ctypes.c_int32 * 2)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_ if k != "reserved"}


class PairInfo(ctypes.Structure):
    _fields_ = [("algo", ctypes.c_int32), ("tile_m", ctypes.c_int32), ("warps", ctypes.c_int32),
                ("strips", ctypes.c_int32), ("bands", ctypes.c_int32), ("braid_cutoff", ctypes.c_int32),
                ("stripes", ctypes.c_int32), ("cols_per_step", ctypes.c_int32), ("reserved", ctypes.c_int32 * 8)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_ if k != "reserved"}


PAIR_DTYPE = np.dtype([("a_offset", np.int64), ("b_offset", np.int64), ("out_offset", np.int64),
                       ("m", np.int32), ("n", np.int32)])

_LIB = None
_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64


def lib():
    """Load libslcs.so; raise if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libslcs.so not found at {LIB_PATH}: run __graft_entry__.build() "
                               f"(make -C platform-independent-lcs_b200)")
        L = ctypes.CDLL(LIB_PATH)
        L.slcs_last_error.restype = ctypes.c_char_p
        L.slcs_status_string.restype = ctypes.c_char_p
        L.slcs_status_string.argtypes = [_i32]
        L.slcs_device_status.argtypes = [_i32, _i32]
        L.slcs_version.restype = _i32
        L.slcs_comb_pair.argtypes = [_vp, _i32, _vp, _i32, _vp, _vp, ctypes.POINTER(Config), _vp]
        L.slcs_comb_pair_host.argtypes = [_vp, _i32, _vp, _i32, _vp, _vp, ctypes.POINTER(Config)]
        L.slcs_comb_batch.argtypes = [_vp, _i32, _vp, _vp, _vp, ctypes.POINTER(Config), _vp]
        L.slcs_comb_batch_host.argtypes = [_vp, _i32, _vp, _i64, _vp, _i64, _vp, _i64, ctypes.POINTER(Config)]
        L.slcs_batch_plan_create.argtypes = [ctypes.POINTER(_vp), _vp, _i32, ctypes.POINTER(Config)]
        L.slcs_batch_plan_run.argtypes = [_vp, _vp, _vp, _vp, _vp]
        L.slcs_batch_plan_destroy.argtypes = [_vp]
        L.slcs_batch_plan_run_host.argtypes = [_vp, _vp, _i64, _vp, _i64, _vp, _i64, _vp]
        L.slcs_batch_plan_run_host16.argtypes = [_vp, _vp, _i64, _vp, _i64, _vp, _i64, _vp]
        L.slcs_batch_plan_launches.argtypes = [_vp]
        L.slcs_batch_plan_launches.restype = _i32
        L.slcs_batch_plan_info.argtypes = [_vp, ctypes.POINTER(PlanInfo)]
        L.slcs_pair_plan_info.argtypes = [_i32, _i32, ctypes.POINTER(Config), ctypes.POINTER(PairInfo)]
        L.slcs_pair_plan_info_sms.argtypes = [_i32, _i32, ctypes.POINTER(Config), _i32, ctypes.POINTER(PairInfo)]
        L.slcs_strands_to_permutation.argtypes = [_vp, _i32, _vp, _i32, _vp, _vp, _vp]
        L.slcs_permutation_to_strands.argtypes = [_vp, _i32, _i32, _vp, _vp, _vp]
        L.slcs_substring_llcs.argtypes = [_vp, _i32, _i32, _vp, _vp, _i32, _vp, _vp]
        L.slcs_permutation_hash.argtypes = [_vp, _i32]
        L.slcs_permutation_hash.restype = _i64
        L.slcs_probe_int_rates.argtypes = [_i32, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), _vp]
        L.slcs_braid_multiply.argtypes = [_vp, _i32, _vp, _i32, _i32, _i32, _vp, ctypes.POINTER(Config), _vp]
        L.slcs_probe_wait_expiry.argtypes = [_i32, _vp]
        L.slcs_strands_hash.argtypes = [_vp, _i32, _vp, _i32, _vp, _vp]
        L.slcs_batch_plan_hash.argtypes = [_vp, _vp, _vp, _vp]
        L.slcs_symbols_to_bytes.argtypes = [_vp, _i32, _vp, _i32, _vp, _vp, _vp, _vp]
        L.slcs_comb_pair_words_host.argtypes = [_vp, _i32, _vp, _i32, _vp, _vp, ctypes.POINTER(Config)]
        L.slcs_comb_pair_noalloc.argtypes = [_vp, _i32, _vp, _i32, _vp, ctypes.POINTER(Config), _vp]
        _LIB = L
    return _LIB


def check(status: int):
    if status != 0:
        msg = lib().slcs_last_error().decode(errors="replace")
        raise SlcsError(status, msg)


def _cfg(cfg: Optional[Config]):
    return ctypes.byref(cfg) if cfg is not None else None


def _stream(stream) -> Optional[int]:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _dptr(t) -> int:
    return t.data_ptr() if t is not None and t.numel() > 0 else 0


def device_status(device: int = 0, clear: bool = True):
    check(lib().slcs_device_status(device, int(clear)))


# ---------------------------------------------------------------------------
# combing
# ---------------------------------------------------------------------------

def comb_pair(a, b, cfg: Optional[Config] = None, stream=None, out=None):
    """Strands of one pair.  a, b: uint8 CUDA tensors.  Returns (h, v) int32
    CUDA views into one contiguous buffer (h first, as the C ABI lays it out)."""
    import torch
    m, n = int(a.numel()), int(b.numel())
    if out is None:
        out = torch.empty(m + n, dtype=torch.int32, device=a.device)
    h, v = out[:m], out[m:]
    check(lib().slcs_comb_pair(_dptr(a), m, _dptr(b), n, _dptr(out), _dptr(out) + 4 * m if n else 0,
                               _cfg(cfg), _stream(stream)))
    return h, v


def pair_plan_info(m: int, n: int, cfg: Optional[Config] = None, sms: Optional[int] = None) -> dict:
    """How comb_pair combs an m x n pair under cfg (kernel family, rows per
    lane, warps, strips, bands, braid cutoff, stripes, columns per step);
    launches nothing.  With `sms`, plans for a device of that many SMs and
    needs no device at all."""
    pi = PairInfo()
    if sms is None:
        check(lib().slcs_pair_plan_info(int(m), int(n), _cfg(cfg), ctypes.byref(pi)))
    else:
        check(lib().slcs_pair_plan_info_sms(int(m), int(n), _cfg(cfg), int(sms), ctypes.byref(pi)))
    return pi.as_dict()


def comb_pair_host(a: np.ndarray, b: np.ndarray, cfg: Optional[Config] = None):
    """Strands of one pair from host numpy arrays (synchronous)."""
    a = np.ascontiguousarray(a, np.uint8)
    b = np.ascontiguousarray(b, np.uint8)
    h = np.empty(len(a), np.int32)
    v = np.empty(len(b), np.int32)
    check(lib().slcs_comb_pair_host(a.ctypes.data, len(a), b.ctypes.data, len(b), h.ctypes.data,
                                    v.ctypes.data, _cfg(cfg)))
    return h, v


def comb_pair_words_host(a: np.ndarray, b: np.ndarray, cfg: Optional[Config] = None):
    """Strands of one pair of Word symbols (any int32 values, at most 256
    distinct) from host numpy arrays; the symbols become bytes on the device."""
    a = np.ascontiguousarray(a, np.int32)
    b = np.ascontiguousarray(b, np.int32)
    h = np.empty(len(a), np.int32)
    v = np.empty(len(b), np.int32)
    check(lib().slcs_comb_pair_words_host(a.ctypes.data, len(a), b.ctypes.data, len(b), h.ctypes.data,
                                          v.ctypes.data, _cfg(cfg)))
    return h, v


def symbols_to_bytes(a, b, stream=None):
    """(a_bytes, b_bytes, alphabet) of int32 CUDA tensors of Word symbols;
    alphabet is the number of distinct symbols, or -1 above 256."""
    import torch
    m, n = int(a.numel()), int(b.numel())
    ab = torch.empty(m, dtype=torch.uint8, device=a.device)
    bb = torch.empty(n, dtype=torch.uint8, device=a.device)
    alpha = torch.empty(1, dtype=torch.int32, device=a.device)
    check(lib().slcs_symbols_to_bytes(_dptr(a), m, _dptr(b), n, _dptr(ab), _dptr(bb), alpha.data_ptr(),
                                      _stream(stream)))
    return ab, bb, int(alpha.item())


_HOST = None


def host_lib():
    """libslcs_host.so: the C++ mirror of the reference interface."""
    global _HOST
    if _HOST is None:
        lib()
        if not os.path.exists(HOST_LIB_PATH):
            raise RuntimeError(f"libslcs_host.so not found at {HOST_LIB_PATH}")
        H = ctypes.CDLL(HOST_LIB_PATH)
        H.slcs_host_run_procedure.argtypes = [ctypes.c_char_p, ctypes.c_char_p, _vp, _i32, _vp, _i32, _vp, _vp,
                                              _vp, _vp, ctypes.c_char_p, _i32]
        H.slcs_host_run_procedure.restype = _i32
        _HOST = H
    return _HOST


def run_procedure(name: str, a: np.ndarray, b: np.ndarray, device_type: str = "gpu"):
    """Run a registered procedure through the C++ mirror of the reference's
    registry: (status, h, v, length_of_lcs, hash, message)."""
    a = np.ascontiguousarray(a, np.int32)
    b = np.ascontiguousarray(b, np.int32)
    h = np.empty(len(a), np.int32)
    v = np.empty(len(b), np.int32)
    llcs = ctypes.c_int32(-1)
    hv = ctypes.c_int64(0)
    err = ctypes.create_string_buffer(512)
    rc = host_lib().slcs_host_run_procedure(name.encode(), device_type.encode(), a.ctypes.data, len(a),
                                            b.ctypes.data, len(b), h.ctypes.data, v.ctypes.data,
                                            ctypes.addressof(llcs), ctypes.addressof(hv), err, len(err))
    return int(rc), h, v, int(llcs.value), int(hv.value), err.value.decode(errors="replace")


def pair_descs(batch) -> np.ndarray:
    """slcs_pair_desc array for a workloads.Batch (strands packed h then v)."""
    off, _ = batch.strand_offsets()
    d = np.zeros(batch.npairs, PAIR_DTYPE)
    d["a_offset"] = batch.a_off
    d["b_offset"] = batch.b_off
    d["out_offset"] = off
    d["m"] = batch.ms
    d["n"] = batch.ns
    return d


class BatchPlan:
    """Reusable schedule of one batch (C ABI slcs_batch_plan)."""

    def __init__(self, descs: np.ndarray, cfg: Optional[Config] = None):
        self._descs = np.ascontiguousarray(descs, PAIR_DTYPE)
        self._h = _vp()
        check(lib().slcs_batch_plan_create(ctypes.byref(self._h), self._descs.ctypes.data, len(self._descs),
                                           _cfg(cfg)))

    @property
    def launches(self) -> int:
        return int(lib().slcs_batch_plan_launches(self._h))

    @property
    def info(self) -> dict:
        pi = PlanInfo()
        check(lib().slcs_batch_plan_info(self._h, ctypes.byref(pi)))
        return pi.as_dict()

    def run(self, a_blob, b_blob, out, stream=None):
        check(lib().slcs_batch_plan_run(self._h, _dptr(a_blob), _dptr(b_blob), _dptr(out), _stream(stream)))

    def run_host(self, a_blob: np.ndarray, b_blob: np.ndarray, out: np.ndarray, stream=None):
        """Host buffers in and out (pinned buffers make the copies asynchronous)."""
        check(lib().slcs_batch_plan_run_host(self._h, a_blob.ctypes.data, a_blob.size, b_blob.ctypes.data,
                                             b_blob.size, out.ctypes.data, out.size, _stream(stream)))

    def hashes(self, out, stream=None):
        """PermutationMatrix::hash of every pair's strands in the plan's output
        blob `out` (int32 CUDA tensor), computed on the device: an int64
        CUDA tensor with one hash per pair."""
        import torch
        h = torch.empty(len(self._descs), dtype=torch.int64, device=out.device)
        check(lib().slcs_batch_plan_hash(self._h, _dptr(out), _dptr(h), _stream(stream)))
        return h

    def run_host16(self, a_blob: np.ndarray, b_blob: np.ndarray, out: np.ndarray, stream=None):
        """As run_host with int16 strands in `out` (pairs with m + n <= 32767)."""
        assert out.dtype == np.int16
        check(lib().slcs_batch_plan_run_host16(self._h, a_blob.ctypes.data, a_blob.size, b_blob.ctypes.data,
                                               b_blob.size, out.ctypes.data, out.size, _stream(stream)))

    def close(self):
        if self._h:
            lib().slcs_batch_plan_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def comb_batch(descs: np.ndarray, a_blob, b_blob, out, cfg: Optional[Config] = None, stream=None):
    descs = np.ascontiguousarray(descs, PAIR_DTYPE)
    check(lib().slcs_comb_batch(descs.ctypes.data, len(descs), _dptr(a_blob), _dptr(b_blob), _dptr(out),
                                _cfg(cfg), _stream(stream)))


def comb_batch_host(descs: np.ndarray, a_blob: np.ndarray, b_blob: np.ndarray, out_len: int,
                    cfg: Optional[Config] = None, out: Optional[np.ndarray] = None) -> np.ndarray:
    descs = np.ascontiguousarray(descs, PAIR_DTYPE)
    a_blob = np.ascontiguousarray(a_blob, np.uint8)
    b_blob = np.ascontiguousarray(b_blob, np.uint8)
    if out is None:
        out = np.empty(out_len, np.int32)
    check(lib().slcs_comb_batch_host(descs.ctypes.data, len(descs), a_blob.ctypes.data, len(a_blob),
                                     b_blob.ctypes.data, len(b_blob), out.ctypes.data, out_len, _cfg(cfg)))
    return out


# ---------------------------------------------------------------------------
# permutation matrix and braid multiplication
# ---------------------------------------------------------------------------

def strands_to_permutation(h, v, stream=None):
    import torch
    m, n = int(h.numel()), int(v.numel())
    r2c = torch.empty(m + n, dtype=torch.int32, device=h.device)
    c2r = torch.empty(m + n, dtype=torch.int32, device=h.device)
    check(lib().slcs_strands_to_permutation(_dptr(h), m, _dptr(v), n, _dptr(r2c), _dptr(c2r), _stream(stream)))
    return r2c, c2r


def permutation_to_strands(r2c, m: int, stream=None):
    """(h, v) strands of P(a, b) from its row -> col array (size m + n)."""
    import torch
    size = int(r2c.numel())
    n = size - int(m)
    out = torch.empty(size, dtype=torch.int32, device=r2c.device)
    check(lib().slcs_permutation_to_strands(_dptr(r2c), int(m), n, _dptr(out), _dptr(out) + 4 * int(m) if n else 0,
                                            _stream(stream)))
    return out[:m], out[m:]


def substring_llcs(v, m: int, begin, end, stream=None):
    """LLCS(a, b[begin[q], end[q])) for every query q, from the v strands of
    the comb of (a, b) (int32 CUDA tensors; -1 for a query out of range)."""
    import torch
    nq = int(begin.numel())
    out = torch.empty(nq, dtype=torch.int32, device=v.device)
    check(lib().slcs_substring_llcs(_dptr(v), int(m), int(v.numel()), _dptr(begin), _dptr(end), nq, _dptr(out),
                                    _stream(stream)))
    return out


def strands_hash(h, v, stream=None) -> int:
    """PermutationMatrix::hash of FromStrands(h, v) computed on the device."""
    import torch
    out = torch.empty(1, dtype=torch.int64, device=h.device)
    check(lib().slcs_strands_hash(_dptr(h), int(h.numel()), _dptr(v), int(v.numel()), out.data_ptr(),
                                  _stream(stream)))
    return int(out.item())


def permutation_hash(col_to_row: np.ndarray) -> int:
    c = np.ascontiguousarray(col_to_row, np.int32)
    return int(lib().slcs_permutation_hash(c.ctypes.data, len(c)))


def braid_multiply(p_r2c, q_r2c, k: int, row_glue: bool, cfg: Optional[Config] = None, stream=None):
    import torch
    size = int(p_r2c.numel()) + int(q_r2c.numel()) - int(k)
    out = torch.empty(size, dtype=torch.int32, device=p_r2c.device)
    check(lib().slcs_braid_multiply(_dptr(p_r2c), int(p_r2c.numel()), _dptr(q_r2c), int(q_r2c.numel()), int(k),
                                    int(bool(row_glue)), _dptr(out), _cfg(cfg), _stream(stream)))
    return out


def probe_int_rates(iters: int = 4096, stream=None):
    """(INT32 min/max ops per second, register-only cell updates per second)."""
    ops = ctypes.c_double()
    cells = ctypes.c_double()
    check(lib().slcs_probe_int_rates(int(iters), ctypes.byref(ops), ctypes.byref(cells), _stream(stream)))
    return ops.value, cells.value


def probe_wait_expiry(wait_ms: int = 200, stream=None):
    """Enqueue the bounded-wait check (a stripe whose producer never runs);
    after a synchronise, device_status() raises SlcsError with status 4."""
    check(lib().slcs_probe_wait_expiry(int(wait_ms), _stream(stream)))
