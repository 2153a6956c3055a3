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

# The variants the autotuner times and the model ranks.  Variant 0 is what the
# library does when nothing is configured (the fixed heuristic).
VARIANTS: List[dict] = [
    {"name": "stream_auto", "cfg": {}},
    {"name": "stream_tn8_32", "cfg": {"strand_bits": 32}},
    {"name": "stream_tn4_32", "cfg": {"strand_bits": 32, "tile_n": 4}},
    {"name": "stream_auto_bpsm2", "cfg": {"blocks_per_sm": 2}},
    {"name": "stream_tn8_32_bpsm2", "cfg": {"strand_bits": 32, "blocks_per_sm": 2}},
    {"name": "wavefront_tm2", "cfg": {"algo": 1, "tile_m": 2}},
    {"name": "wavefront_tm4", "cfg": {"algo": 1, "tile_m": 4}},
    {"name": "wavefront_tm8", "cfg": {"algo": 1, "tile_m": 8}},
    {"name": "wavefront_tm16", "cfg": {"algo": 1, "tile_m": 16}},
    {"name": "wavefront_tm16_w8", "cfg": {"algo": 1, "tile_m": 16, "warps": 8}},
    {"name": "wavefront_tm8_w8", "cfg": {"algo": 1, "tile_m": 8, "warps": 8}},
]
HEURISTIC = 0
PLAIN = 7  # the plain wavefront kernel with its default tile


def variant_config(i: int, use_graph: bool = True) -> Config:
    kw = dict(VARIANTS[i]["cfg"])
    if use_graph:
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
        return np.argmin(self.predict(X), axis=1)

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


def ranking(batch) -> Optional[np.ndarray]:
    """Variant indices, fastest predicted first (None without a model)."""
    model = installed_model()
    if model is None:
        return None
    return np.argsort(model.predict(batch_features(batch)[None, :])[0], kind="stable")


def choose(batch) -> Optional[Config]:
    """The model's variant for a batch, or None when no model is installed."""
    r = ranking(batch)
    return None if r is None else variant_config(int(r[0]))
