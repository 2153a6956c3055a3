"""The learned cost model: an FP32 MLP (4 -> 64 -> 64 -> K) that predicts the
log2 run time of K kernel variants for a batch shape, trained and evaluated on
the GPU through the C ABI (kernels in csrc/costmodel.cu).

Features of a batch: log2 of its median m, median n, alphabet size (distinct
symbols, at least 2) and number of pairs.  The planner picks the variant with
the smallest predicted time; the fixed heuristic (variant 0, the library's
default rule) is the fallback whenever no trained model is installed.  The
model chooses launch parameters only; every variant yields identical strands.
"""
from __future__ import annotations

import ctypes
import json
import math
import os
from typing import List, Optional

import numpy as np

from . import Config, check, lib

HERE = os.path.dirname(os.path.abspath(__file__))
MODEL_PATH = os.path.join(HERE, "data", "costmodel.json")
DB_PATH = os.path.join(HERE, "data", "timings.npz")

# The variants the autotuner times and the model ranks.  "batch" variants are
# launch plans of one batch (slcs_batch_plan_*); "pair" variants comb each
# pair of a shape with slcs_comb_pair under a tiling and a steady-ant cutoff
# (src/braid_multiplication.hpp:204-270 is the recursion whose base case the
# cutoff moves), and apply to shapes of at most PAIR_BATCH_MAX pairs.
# Variant 0 is what the library does for a batch when nothing is configured.
PAIR_BATCH_MAX = 8
VARIANTS: List[dict] = [
    {"name": "stream_auto", "kind": "batch", "cfg": {}},
    {"name": "stream_tn8_32", "kind": "batch", "cfg": {"strand_bits": 32}},
    {"name": "stream_tn4_32", "kind": "batch", "cfg": {"strand_bits": 32, "tile_n": 4}},
    {"name": "stream_auto_bpsm4", "kind": "batch", "cfg": {"blocks_per_sm": 4}},
    {"name": "stream_tn8_32_bpsm2", "kind": "batch", "cfg": {"strand_bits": 32, "blocks_per_sm": 2}},
    {"name": "wavefront_tm2", "kind": "batch", "cfg": {"algo": 1, "tile_m": 2}},
    {"name": "wavefront_tm4", "kind": "batch", "cfg": {"algo": 1, "tile_m": 4}},
    {"name": "wavefront_tm8", "kind": "batch", "cfg": {"algo": 1, "tile_m": 8}},
    {"name": "wavefront_tm16", "kind": "batch", "cfg": {"algo": 1, "tile_m": 16}},
    {"name": "wavefront_tm16_w8", "kind": "batch", "cfg": {"algo": 1, "tile_m": 16, "warps": 8}},
    {"name": "wavefront_tm8_w8", "kind": "batch", "cfg": {"algo": 1, "tile_m": 8, "warps": 8}},
] + [
    {"name": f"pair_auto_c{c}", "kind": "pair", "cfg": {"braid_cutoff": c}} for c in (64, 256, 1024, 4096)
] + [
    {"name": f"pair_strips{s}_c{c}", "kind": "pair", "cfg": {"algo": 2, "strips": s, "bands": 1, "braid_cutoff": c}}
    for s in (2, 4, 8, 16) for c in (256, 1024)
] + [
    {"name": f"pair_bands{r}_c{c}", "kind": "pair", "cfg": {"algo": 2, "strips": 1, "bands": r, "braid_cutoff": c}}
    for r in (2, 4, 8) for c in (256, 1024)
]
HEURISTIC = 0
PLAIN = 7  # the plain wavefront kernel with its default tile
PAIR_DEFAULT = [v["name"] for v in VARIANTS].index("pair_auto_c256")  # the library's rule for one pair


def is_pair(i: int) -> bool:
    return VARIANTS[i]["kind"] == "pair"


def applicable(batch: float) -> np.ndarray:
    """Which variants apply to a shape of `batch` pairs (pair variants comb
    the pairs one call each, so they are offered for small batches only)."""
    return np.array([not is_pair(i) or batch <= PAIR_BATCH_MAX for i in range(len(VARIANTS))])


def variant_config(i: int, use_graph: bool = True) -> Config:
    kw = dict(VARIANTS[i]["cfg"])
    if use_graph and not is_pair(i):
        kw["use_graph"] = 1
    return Config.make(**kw)


def features_of(m: float, n: float, sigma: float, batch: float) -> np.ndarray:
    return np.array([math.log2(max(m, 1)), math.log2(max(n, 1)), math.log2(max(sigma, 2)),
                     math.log2(max(batch, 1))], np.float32)


def batch_features(batch) -> np.ndarray:
    """Features of a workloads.Batch."""
    if batch.npairs == 0:
        return features_of(1, 1, 2, 1)
    sample = batch.a_blob[: min(len(batch.a_blob), 1 << 20)]
    sigma = len(np.unique(sample))
    return features_of(float(np.median(batch.ms)), float(np.median(batch.ns)), sigma, batch.npairs)


_f = ctypes.POINTER(ctypes.c_float)
_u8 = ctypes.POINTER(ctypes.c_uint8)


def _ptr(a, t):
    return a.ctypes.data_as(t)


def _bind():
    L = lib()
    if not getattr(L, "_cm_bound", False):
        L.slcs_costmodel_param_count.argtypes = [ctypes.c_int32]
        L.slcs_costmodel_param_count.restype = ctypes.c_int32
        L.slcs_costmodel_init.argtypes = [_f, ctypes.c_int32, ctypes.c_uint64, _f, _f]
        L.slcs_costmodel_train.argtypes = [_f, ctypes.c_int32, _f, _f, _u8, ctypes.c_int32, ctypes.c_int32,
                                           ctypes.c_float, _f]
        L.slcs_costmodel_predict.argtypes = [_f, ctypes.c_int32, _f, ctypes.c_int32, _f]
        L.slcs_costmodel_grad.argtypes = [_f, ctypes.c_int32, _f, _f, _u8, ctypes.c_int32, _f, _f]
        L._cm_bound = True
    return L


def param_count(k: int) -> int:
    return int(_bind().slcs_costmodel_param_count(k))


def init_params(k: int, X: np.ndarray, seed: int = 0) -> np.ndarray:
    X = np.asarray(X, np.float32)
    mean = np.ascontiguousarray(X.mean(0), np.float32)
    std = np.ascontiguousarray(X.std(0) + 1e-3, np.float32)
    p = np.zeros(param_count(k), np.float32)
    check(_bind().slcs_costmodel_init(_ptr(p, _f), k, seed, _ptr(mean, _f), _ptr(std, _f)))
    return p


def train(params: np.ndarray, X, T, M, epochs: int = 2000, lr: float = 3e-3) -> float:
    """Full-batch Adam on the GPU; updates params in place, returns the loss."""
    k = T.shape[1]
    X = np.ascontiguousarray(X, np.float32)
    T = np.ascontiguousarray(T, np.float32)
    M = np.ascontiguousarray(M, np.uint8)
    loss = ctypes.c_float()
    check(_bind().slcs_costmodel_train(_ptr(params, _f), k, _ptr(X, _f), _ptr(T, _f), _ptr(M, _u8), len(X),
                                       int(epochs), float(lr), ctypes.byref(loss)))
    return float(loss.value)


def predict(params: np.ndarray, k: int, X) -> np.ndarray:
    X = np.ascontiguousarray(X, np.float32).reshape(-1, 4)
    Y = np.empty((len(X), k), np.float32)
    check(_bind().slcs_costmodel_predict(_ptr(np.ascontiguousarray(params, np.float32), _f), k, _ptr(X, _f),
                                         len(X), _ptr(Y, _f)))
    return Y


def gradient(params: np.ndarray, X, T, M):
    k = T.shape[1]
    X = np.ascontiguousarray(X, np.float32)
    T = np.ascontiguousarray(T, np.float32)
    M = np.ascontiguousarray(M, np.uint8)
    g = np.zeros_like(params)
    loss = ctypes.c_float()
    check(_bind().slcs_costmodel_grad(_ptr(np.ascontiguousarray(params, np.float32), _f), k, _ptr(X, _f),
                                      _ptr(T, _f), _ptr(M, _u8), len(X), _ptr(g, _f), ctypes.byref(loss)))
    return float(loss.value), g


class CostModel:
    def __init__(self, params: np.ndarray, variants: List[str]):
        self.params = np.ascontiguousarray(params, np.float32)
        self.variants = list(variants)

    @property
    def k(self) -> int:
        return len(self.variants)

    def predict(self, X) -> np.ndarray:
        return predict(self.params, self.k, X)

    def choose_index(self, X) -> np.ndarray:
        """Fastest predicted applicable variant per row of X (features; the
        batch size is 2 ** X[:, 3])."""
        X = np.asarray(X, np.float32).reshape(-1, 4)
        Y = self.predict(X)
        ok = np.stack([applicable(2.0 ** float(x[3])) for x in X])
        return np.argmin(np.where(ok, Y, np.inf), axis=1)

    def save(self, path: str = MODEL_PATH, extra: Optional[dict] = None):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        d = {"variants": self.variants, "params": [float(x) for x in self.params]}
        if extra:
            d.update(extra)
        with open(path, "w") as f:
            json.dump(d, f)

    @classmethod
    def load(cls, path: str = MODEL_PATH) -> Optional["CostModel"]:
        if not os.path.exists(path):
            return None
        with open(path) as f:
            d = json.load(f)
        names = [v["name"] for v in VARIANTS]
        if d.get("variants") != names:
            return None  # trained for another variant list
        return cls(np.array(d["params"], np.float32), d["variants"])


_MODEL = None


def installed_model() -> Optional[CostModel]:
    global _MODEL
    if _MODEL is None:
        _MODEL = CostModel.load() or False
    return _MODEL or None


def ranking(batch, kind: Optional[str] = None) -> Optional[np.ndarray]:
    """Applicable variant indices (of `kind` "batch" or "pair" when given),
    fastest predicted first (None without a model)."""
    model = installed_model()
    if model is None:
        return None
    x = batch_features(batch)
    order = np.argsort(model.predict(x[None, :])[0], kind="stable")
    ok = applicable(batch.npairs)
    return np.array([int(i) for i in order if ok[i] and (kind is None or VARIANTS[int(i)]["kind"] == kind)])


def choose(batch) -> Optional[Config]:
    """The model's batch-plan variant for a batch, or None when no model is installed."""
    r = ranking(batch, kind="batch")
    return None if r is None else variant_config(int(r[0]))
