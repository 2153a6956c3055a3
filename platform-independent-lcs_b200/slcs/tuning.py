"""Variant selection for batches and the secondary measurements of bench.py.

choose_batch_config() asks the trained cost model when one is available
(slcs.costmodel) and otherwise falls back to the fixed heuristic.  The model
only picks launch parameters; every variant produces identical strands.
"""
from __future__ import annotations

import json
import os
import time

import numpy as np

from . import Config, check, lib, strands_to_permutation, permutation_hash

HERE = os.path.dirname(os.path.abspath(__file__))


def heuristic_batch_config(batch) -> Config:
    """The library's fixed rule (stream mode, 16-lane segments, the smallest
    rows-per-lane whose segment holds nine pairs in ten whole)."""
    return Config.make(use_graph=1)


def choose_batch_config(batch):
    try:
        from . import costmodel
        cfg = costmodel.choose(batch)
        if cfg is not None:
            return cfg, "cost_model"
    except Exception:
        pass
    return heuristic_batch_config(batch), "heuristic"


def per_pair_loop(batch, a_d, b_d, out, stream_handle, limit=None):
    """The plain path: one slcs_comb_pair launch per pair, device pointers."""
    L = lib()
    A, B, O_ = a_d.data_ptr(), b_d.data_ptr(), out.data_ptr()
    from . import pair_descs
    d = pair_descs(batch)
    n = batch.npairs if limit is None else min(limit, batch.npairs)
    for p in range(n):
        m, nn = int(d["m"][p]), int(d["n"][p])
        o = O_ + 4 * int(d["out_offset"][p])
        check(L.slcs_comb_pair(A + int(d["a_offset"][p]), m, B + int(d["b_offset"][p]), nn, o, o + 4 * m, None,
                               stream_handle))


def secondary_measurements(batch, a_d, b_d, out, roof_gcups, dev):
    import torch
    res = {}
    st = torch.cuda.current_stream()
    # plain per-pair launch loop over the same batch
    per_pair_loop(batch, a_d, b_d, out, st.cuda_stream, limit=200)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(st)
    per_pair_loop(batch, a_d, b_d, out, st.cuda_stream)
    e1.record(st)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    ms = e0.elapsed_time(e1)
    res["plain_per_pair"] = {"gcups": batch.cells / (ms * 1e-3) / 1e9, "ms": ms, "wall_ms": wall * 1e3,
                             "launches": batch.npairs}
    # the 2^20 x 2^20 pair: roofline fraction of the wavefront kernel
    from . import workloads as W
    a, b = W.pair_1m()
    ad = torch.from_numpy(a).to(dev)
    bd = torch.from_numpy(b).to(dev)
    o = torch.empty(len(a) + len(b), dtype=torch.int32, device=dev)
    from . import comb_pair
    cfg = Config.make()  # default rule: 16 rows per lane, 8 warps per block at this height
    comb_pair(ad, bd, cfg=cfg, out=o)
    torch.cuda.synchronize()
    e0.record(st)
    comb_pair(ad, bd, cfg=cfg, out=o)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    cells = len(a) * len(b)
    g = cells / (ms * 1e-3) / 1e9
    _, c2r = strands_to_permutation(o[:len(a)], o[len(a):])
    hv = permutation_hash(c2r.cpu().numpy())
    gold = None
    try:
        gold = json.load(open(os.path.join(HERE, "..", "..", "tests", "golden", "golden.json")))["pair_1M"]["hash"]
    except Exception:
        pass
    res["long_pair"] = {"workload": "pair_1M (1048576 x 1048576, uniform {0..3})", "ms": ms, "gcups": g,
                        "roofline_frac": g / roof_gcups, "hash": hv,
                        "bitexact_vs_reference": (hv == gold) if gold is not None else None,
                        "variant": {"tile_m": 16, "warps": 8}}
    return res
