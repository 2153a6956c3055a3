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


def choose_batch_config(batch, timer=None, top: int = 3):
    """(config, how it was chosen, details).

    With a trained cost model, its first choice -- or, when `timer` is given
    (a callable that times one run of a Config on the actual batch), the
    fastest of its `top` best-ranked variants, measured: the model prunes the
    search from every variant to a few.  Without a model, the fixed
    heuristic."""
    try:
        from . import costmodel
        order = costmodel.ranking(batch, kind="batch")
    except Exception:
        order = None
    if order is None:
        return heuristic_batch_config(batch), "heuristic", {}
    names = [costmodel.VARIANTS[int(i)]["name"] for i in order[:top]]
    if timer is None:
        return costmodel.variant_config(int(order[0])), "cost_model", {"model_choice": names[0]}
    times = {}
    for i in order[:top]:
        times[costmodel.VARIANTS[int(i)]["name"]] = float(timer(costmodel.variant_config(int(i))))
    best = min(times, key=times.get)
    idx = [v["name"] for v in costmodel.VARIANTS].index(best)
    return (costmodel.variant_config(idx), f"cost_model_top{top}_timed",
            {"model_choice": names[0], "candidates_ms": times, "chosen": best})


def choose_pair_config(m: int, n: int, sigma: int, timer=None, top: int = 3):
    """(config, how it was chosen, details) for one m x n pair: the cost
    model's best-ranked single-pair variant (tiling and steady-ant cutoff), or
    with `timer` the fastest of its `top` best-ranked ones, measured; without
    a model, the library's own rule (Config())."""
    from . import costmodel
    model = costmodel.installed_model()
    if model is None:
        return Config.make(), "library_rule", {}
    y = model.predict(costmodel.features_of(m, n, sigma, 1)[None, :])[0]
    order = [int(i) for i in np.argsort(y, kind="stable") if costmodel.is_pair(int(i))]
    names = [costmodel.VARIANTS[i]["name"] for i in order[:top]]
    if timer is None:
        return costmodel.variant_config(order[0]), "cost_model", {"model_choice": names[0]}
    times = {costmodel.VARIANTS[i]["name"]: float(timer(costmodel.variant_config(i))) for i in order[:top]}
    best = min(times, key=times.get)
    idx = [v["name"] for v in costmodel.VARIANTS].index(best)
    return (costmodel.variant_config(idx), f"cost_model_top{top}_timed",
            {"model_choice": names[0], "candidates_ms": times, "chosen": best})


def per_pair_loop(batch, a_d, b_d, out, stream_handle, limit=None):
    """The plain path as a caller would write it: one slcs_comb_pair call per
    pair, device pointers (each call plans, allocates its scratch, launches
    and frees)."""
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


def per_pair_loop_lean(batch, a_d, b_d, out, stream_handle, limit=None):
    """The plain path at its leanest: one wavefront launch per pair on
    preallocated scratch (slcs_comb_pair_noalloc: a counter reset and the
    kernel, nothing planned or allocated per pair)."""
    L = lib()
    A, B, O_ = a_d.data_ptr(), b_d.data_ptr(), out.data_ptr()
    from . import pair_descs
    d = pair_descs(batch)
    n = batch.npairs if limit is None else min(limit, batch.npairs)
    f = L.slcs_comb_pair_noalloc
    for p in range(n):
        m, nn = int(d["m"][p]), int(d["n"][p])
        check(f(A + int(d["a_offset"][p]), m, B + int(d["b_offset"][p]), nn, O_ + 4 * int(d["out_offset"][p]),
                None, stream_handle))


def _golden():
    try:
        with open(os.path.join(HERE, "..", "..", "tests", "golden", "golden.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def _time_loop(loop, batch, a_d, b_d, out, st):
    import torch
    loop(batch, a_d, b_d, out, st.cuda_stream, limit=200)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(st)
    loop(batch, a_d, b_d, out, st.cuda_stream)
    e1.record(st)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    ms = e0.elapsed_time(e1)
    return {"gcups": batch.cells / (ms * 1e-3) / 1e9, "ms": ms, "wall_ms": wall * 1e3}


def pair_configs(roof_gcups, dev):
    """The 4096 x 4096 uniform pair and the 131072 x 131072 mutated pair under
    the library's default rule: best of five, GCUPS, fraction of the integer
    roofline, and the reference's hash of the permutation."""
    import torch
    from . import comb_pair, pair_plan_info
    from . import workloads as W
    gold = _golden()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    res = {}
    for name, gen, desc in (("pair_4096", W.pair_4096, "4096 x 4096, uniform {0..3}"),
                            ("pair_131072_mutated", W.pair_131072_mutated,
                             "131072 x 131072, b = a with 10% substitutions and 1%+1% indels")):
        a, b = gen()
        ad = torch.from_numpy(a).to(dev)
        bd = torch.from_numpy(b).to(dev)
        o = torch.empty(len(a) + len(b), dtype=torch.int32, device=dev)
        comb_pair(ad, bd, out=o)
        torch.cuda.synchronize()
        runs = []
        for _ in range(5):
            e0.record(st)
            comb_pair(ad, bd, out=o)
            e1.record(st)
            torch.cuda.synchronize()
            runs.append(e0.elapsed_time(e1))
        ms = min(runs)
        g = len(a) * len(b) / (ms * 1e-3) / 1e9
        _, c2r = strands_to_permutation(o[:len(a)], o[len(a):])
        hv = permutation_hash(c2r.cpu().numpy())
        want = gold.get(name, {}).get("hash")
        res[name] = {"workload": desc, "ms": ms, "gcups": g, "roofline_frac": g / roof_gcups, "runs_ms": runs,
                     "hash": hv, "bitexact_vs_reference": (hv == want) if want is not None else None,
                     "variant": pair_plan_info(len(a), len(b))}

        # the cost model's single-pair variant (its three best-ranked, timed)
        def timer(cfg):
            comb_pair(ad, bd, cfg=cfg, out=o)
            torch.cuda.synchronize()
            best = float("inf")
            for _ in range(3):
                e0.record(st)
                comb_pair(ad, bd, cfg=cfg, out=o)
                e1.record(st)
                torch.cuda.synchronize()
                best = min(best, e0.elapsed_time(e1))
            return best

        cfg, how, info = choose_pair_config(len(a), len(b), 4, timer=timer)
        if how != "library_rule":
            tms = min(info["candidates_ms"].values())
            comb_pair(ad, bd, cfg=cfg, out=o)
            _, c2r = strands_to_permutation(o[:len(a)], o[len(a):])
            thv = permutation_hash(c2r.cpu().numpy())
            tg = len(a) * len(b) / (tms * 1e-3) / 1e9
            res[name]["tuned"] = {"ms": tms, "gcups": tg, "roofline_frac": tg / roof_gcups, "how": how,
                                  "tuning": info, "bitexact_vs_reference": (thv == want) if want is not None else None,
                                  "variant": pair_plan_info(len(a), len(b), cfg)}
    return res


def costmodel_block():
    """Regret of the installed cost model on the autotuner's held-out test
    shapes (time of its choice over the fastest measured variant, minus one),
    beside the fixed heuristic and the plain kernel; the model's predictions
    run on the GPU."""
    from . import autotune as AT
    from . import costmodel as CM
    model = CM.installed_model()
    if model is None or not os.path.exists(CM.DB_PATH):
        return None
    import numpy as np
    db = np.load(CM.DB_PATH)
    rep = AT.report(model, db["test_X"], db["test_ms"])
    return {"shapes": int(len(db["test_X"])), "variants": model.k, "variant_names": model.variants,
            "regret": rep, "all_variants_bitexact_on_every_shape": bool(db["test_agree"].all())}


def secondary_measurements(batch, a_d, b_d, out, roof_gcups, dev, sampler=None):
    """Plain per-pair loops, configurations 1 and 2, the 2^20 pair (best of 5
    runs, with the SM clocks sampled while it runs when `sampler` -- a
    context-manager factory with a summary() -- is given), strips and braid
    products, and the cost model's regret."""
    import torch
    res = {}
    st = torch.cuda.current_stream()
    # plain per-pair launch loops over the same batch
    res["plain_per_pair"] = dict(_time_loop(per_pair_loop_lean, batch, a_d, b_d, out, st), launches=2 * batch.npairs,
                                 how="slcs_comb_pair_noalloc per pair: counter reset + one wavefront launch")
    res["plain_per_pair_alloc"] = dict(_time_loop(per_pair_loop, batch, a_d, b_d, out, st), launches=batch.npairs,
                                       how="slcs_comb_pair per pair: plan, allocate, launch, free")
    res["configs"] = pair_configs(roof_gcups, dev)
    try:
        res["costmodel"] = costmodel_block()
    except Exception as e:  # reported, not fatal: the headline does not depend on it
        res["costmodel"] = {"error": str(e)}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the 2^20 x 2^20 pair: roofline fraction of the wavefront kernel
    from . import workloads as W
    a, b = W.pair_1m()
    ad = torch.from_numpy(a).to(dev)
    bd = torch.from_numpy(b).to(dev)
    o = torch.empty(len(a) + len(b), dtype=torch.int32, device=dev)
    from . import comb_pair, pair_plan_info
    cfg = Config.make()  # the library's default rule for a pair of this height
    comb_pair(ad, bd, cfg=cfg, out=o)
    torch.cuda.synchronize()
    runs = []
    smp = sampler() if sampler else None
    if smp:
        smp.__enter__()
    for _ in range(5):
        e0.record(st)
        comb_pair(ad, bd, cfg=cfg, out=o)
        e1.record(st)
        torch.cuda.synchronize()
        runs.append(e0.elapsed_time(e1))
    if smp:
        smp.__exit__(None, None, None)
    ms = min(runs)
    cells = len(a) * len(b)
    g = cells / (ms * 1e-3) / 1e9
    _, c2r = strands_to_permutation(o[:len(a)], o[len(a):])
    hv = permutation_hash(c2r.cpu().numpy())
    gold = _golden().get("pair_1M", {}).get("hash")
    res["long_pair"] = {"workload": "pair_1M (1048576 x 1048576, uniform {0..3})", "ms": ms, "gcups": g,
                        "roofline_frac": g / roof_gcups, "hash": hv,
                        "bitexact_vs_reference": (hv == gold) if gold is not None else None,
                        "variant": pair_plan_info(len(a), len(b), cfg),
                        "runs_ms": runs,
                        "clocks": smp.summary() if smp else None}
    res.update(strips_and_braid(ad, bd, o, gold, dev))
    return res


def _measured_hbm_gbs():
    try:
        with open(os.path.join(HERE, "..", "..", "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json (copy, read+write bytes)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s"


def strips_and_braid(ad, bd, o, gold_hash, dev):
    """The 2^20 x 2^20 pair in the default tiling (row bands glued by
    row-glue braid products) over the cutoff sweep {64, 256, 1024, 4096}; and
    one braid product alone (the top merge of the two halves of b, overlap
    k = 2^20) against HBM."""
    import torch
    from . import braid_multiply, comb_pair, pair_plan_info
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    m, n = int(ad.numel()), int(bd.numel())
    cells = m * n

    def timed(fn, reps=2):
        fn()
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(reps):
            e0.record(st)
            fn()
            e1.record(st)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best

    sweep = {}
    for cutoff in (64, 256, 1024, 4096):
        cfg = Config.make(braid_cutoff=cutoff)
        ms = timed(lambda: comb_pair(ad, bd, cfg=cfg, out=o))
        _, c2r = strands_to_permutation(o[:m], o[m:])
        hv = permutation_hash(c2r.cpu().numpy())
        sweep[str(cutoff)] = {"ms": ms, "gcups": cells / (ms * 1e-3) / 1e9,
                              "bitexact_vs_reference": (hv == gold_hash) if gold_hash is not None else None}
    half = n // 2
    hp, vp = comb_pair(ad, bd[:half])
    hq, vq = comb_pair(ad, bd[half:])
    P = strands_to_permutation(hp, vp)[0]
    Q = strands_to_permutation(hq, vq)[0]
    peak, peak_src = _measured_hbm_gbs()
    braid = {}
    for cutoff in (64, 256, 1024, 4096):
        cfg = Config.make(braid_cutoff=cutoff)
        ms = timed(lambda: braid_multiply(P, Q, m, False, cfg=cfg), reps=3)
        p, q = int(P.numel()), int(Q.numel())
        algo_bytes = 4 * (p + q) + 4 * (p + q - m)
        gbs = algo_bytes / (ms * 1e-3) / 1e9
        braid[str(cutoff)] = {"ms": ms, "algorithmic_bytes": algo_bytes, "achieved_gbs": gbs, "frac": gbs / peak}
    tiles = pair_plan_info(m, n)
    return {"long_pair_tiles": {"workload": f"pair_1M as {tiles['bands']} row bands x {tiles['strips']} column "
                                             "strips + braid merge trees", "cutoff_sweep": sweep},
            "braid_top_merge": {"workload": "staggered_multiply<false>(P(a,b[:n/2]), P(a,b[n/2:]), k=2^20)",
                                "bound": "hbm", "peak_gbs": peak, "peak_source": peak_src, "by_cutoff": braid}}
