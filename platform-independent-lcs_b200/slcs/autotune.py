"""Autotuner: times every kernel variant on generated batch shapes, checks
that all variants agree bit for bit, and keeps the timings as the cost model's
training data.  Also scores a variant chooser by its regret against exhaustive
tuning.  (Whether the variants also agree with the reference's algorithm is
checked by the GPU tests against the CPU oracle, on a sample of these shapes.)

    python -m slcs.autotune collect --train 3000 --test 1000 --out DB.npz
    python -m slcs.autotune collect --train 8000 --train-start 2400 ...   # only shapes 2400.. of the sample
    python -m slcs.autotune merge A.npz B.npz --out DB.npz                # concatenate collections
    python -m slcs.autotune fit DB.npz           # trains on the GPU, writes slcs/data/costmodel.json

Shapes follow the sweep definition (slcs.workloads.sweep_shapes): m, n
log-uniform in [64, 262144], alphabet in {2, 4, 20, 256}, i.i.d. or mutated
content (5 % substitutions), batch log-uniform in [1, 4096], with the batch
cut so that a shape stays under the per-shape cell budget.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import BatchPlan, PAIR_DTYPE, costmodel as CM
from . import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))


def gpu_shape(shape: W.Shape, device):
    """One sweep shape materialised on the GPU: (descs, a, b, total strands)."""
    import torch
    g = torch.Generator(device=device).manual_seed(int(shape.seed))
    B, m, n, s = shape.batch, shape.m, shape.n, shape.sigma
    m16, n16 = (m + 15) // 16 * 16, (n + 15) // 16 * 16
    a = torch.zeros((B, m16), dtype=torch.uint8, device=device)
    a[:, :m] = torch.randint(0, s, (B, m), generator=g, device=device, dtype=torch.int32).to(torch.uint8)
    b = torch.zeros((B, n16), dtype=torch.uint8, device=device)
    if shape.mutated:
        k = min(m, n)
        src = a[:, :k].to(torch.int32)
        sub = torch.rand((B, k), generator=g, device=device) < 0.05
        shift = torch.randint(1, max(s, 2), (B, k), generator=g, device=device, dtype=torch.int32)
        b[:, :k] = torch.where(sub, (src + shift) % s, src).to(torch.uint8)
        if n > k:
            b[:, k:n] = torch.randint(0, s, (B, n - k), generator=g, device=device, dtype=torch.int32).to(torch.uint8)
    else:
        b[:, :n] = torch.randint(0, s, (B, n), generator=g, device=device, dtype=torch.int32).to(torch.uint8)
    d = np.zeros(B, PAIR_DTYPE)
    d["a_offset"] = np.arange(B, dtype=np.int64) * m16
    d["b_offset"] = np.arange(B, dtype=np.int64) * n16
    d["out_offset"] = np.arange(B, dtype=np.int64) * (m + n)
    d["m"] = m
    d["n"] = n
    return d, a.reshape(-1), b.reshape(-1), B * (m + n)


def run_variant(i: int, descs, a, b, out, plan=None):
    """One run of variant i on a materialised shape (device blobs a, b; strands
    into out).  Batch variants run their plan; pair variants comb the pairs
    one slcs_comb_pair call each."""
    from . import comb_pair
    if not CM.is_pair(i):
        plan.run(a, b, out)
        return
    cfg = CM.variant_config(i)
    for d in descs:
        m, n = int(d["m"]), int(d["n"])
        o = int(d["out_offset"])
        comb_pair(a[int(d["a_offset"]):int(d["a_offset"]) + m], b[int(d["b_offset"]):int(d["b_offset"]) + n],
                  cfg=cfg, out=out[o:o + m + n])


def time_variants(descs, a, b, total, reps: int = 2, slow_ms: float = 50.0):
    """Best-of-reps milliseconds of every applicable variant (NaN where a
    variant does not apply), whether all outputs agree, and the output."""
    import torch
    out_ref = None
    times = np.full(len(CM.VARIANTS), np.nan, np.float64)
    ok = CM.applicable(len(descs))
    agree = True
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i in range(len(CM.VARIANTS)):
        if not ok[i]:
            continue
        plan = None if CM.is_pair(i) else BatchPlan(descs, CM.variant_config(i, use_graph=False))
        out = torch.empty(total, dtype=torch.int32, device=a.device)
        e0.record()
        run_variant(i, descs, a, b, out, plan)  # warm-up and result
        e1.record()
        torch.cuda.synchronize()
        warm = e0.elapsed_time(e1)
        best = float("inf")
        for r in range(reps if warm < 10.0 else 1):  # slow variants: one timed run after the warm-up
            e0.record()
            run_variant(i, descs, a, b, out, plan)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
            if best > slow_ms:
                break
        times[i] = best
        if out_ref is None:
            out_ref = out
        elif not torch.equal(out_ref, out):
            agree = False
        if plan is not None:
            plan.close()
    return times, agree, out_ref


def collect(shapes, device, log_every: int = 200, budget_s: float = 0.0):
    """Timings of every applicable variant on every shape, and whether all
    variants produced the same strands; with budget_s > 0, stops after that
    many seconds (the shapes done so far are returned, in order)."""
    import torch
    feats, times, agree_all = [], [], []
    t0 = time.time()
    for j, sh in enumerate(shapes):
        if budget_s > 0 and time.time() - t0 > budget_s:
            print(f"  budget reached after {j} shapes", flush=True)
            break
        descs, a, b, total = gpu_shape(sh, device)
        t, agree, out = time_variants(descs, a, b, total)
        feats.append(CM.features_of(sh.m, sh.n, sh.sigma, sh.batch))
        times.append(t)
        agree_all.append(agree)
        del a, b, out
        if log_every and (j + 1) % log_every == 0:
            print(f"  {j + 1}/{len(shapes)} shapes, {time.time() - t0:.0f} s", flush=True)
        torch.cuda.synchronize()
    return np.array(feats, np.float32), np.array(times, np.float64), np.array(agree_all, bool)


def regret(times: np.ndarray, chosen: np.ndarray) -> dict:
    """Regret of a chooser: time(chosen) / time(best) - 1 per shape, over the
    shapes where the chosen variant was measured."""
    best = np.nanmin(times, axis=1)
    got = times[np.arange(len(times)), chosen]
    keep = np.isfinite(got)
    got, best = got[keep], best[keep]
    r = got / best - 1.0
    return {"shapes": int(keep.sum()), "mean": float(np.mean(r)), "median": float(np.median(r)),
            "p90": float(np.quantile(r, 0.9)),
            "geomean_time_ratio": float(np.exp(np.mean(np.log(got / best)))),
            "total_time_ratio": float(got.sum() / best.sum()), "optimal_share": float(np.mean(r <= 1e-9))}


def training_arrays(feats: np.ndarray, times: np.ndarray):
    T = np.log2(np.where(np.isfinite(times), times, 1.0)).astype(np.float32)
    M = np.isfinite(times).astype(np.uint8)
    return feats.astype(np.float32), T, M


def fit(feats, times, epochs: int = 3000, lr: float = 3e-3, seed: int = 0):
    X, T, M = training_arrays(feats, times)
    k = T.shape[1]
    p = CM.init_params(k, X, seed)
    loss = CM.train(p, X, T, M, epochs=epochs, lr=lr)
    return CM.CostModel(p, [v["name"] for v in CM.VARIANTS]), loss


def report(model: CM.CostModel, feats, times) -> dict:
    """Regret of the model's choices (among the applicable variants), of the
    fixed heuristic (the library's batch default), of the library's
    single-pair rule on the shapes it applies to, and of the plain kernel."""
    chosen = model.choose_index(feats)
    small = np.isfinite(times[:, CM.PAIR_DEFAULT])
    rep = {"model": regret(times, chosen),
           "heuristic": regret(times, np.full(len(times), CM.HEURISTIC)),
           "plain": regret(times, np.full(len(times), CM.PLAIN))}
    if small.any():
        rep["model_small_batches"] = regret(times[small], chosen[small])
        rep["pair_default_small_batches"] = regret(times[small], np.full(int(small.sum()), CM.PAIR_DEFAULT))
        rep["heuristic_small_batches"] = regret(times[small], np.full(int(small.sum()), CM.HEURISTIC))
    return rep


def merge(parts, out):
    """Concatenate collections of the same variant list (train and test parts)."""
    dbs = [np.load(p) for p in parts]
    names = [list(d["variants"]) for d in dbs]
    if any(n != names[0] for n in names):
        raise SystemExit("collections timed different variant lists")
    res = {"variants": dbs[0]["variants"]}
    for split in ("train", "test"):
        for key in ("X", "ms", "agree", "shape"):
            k = f"{split}_{key}"
            res[k] = np.concatenate([d[k] for d in dbs if k in d.files and len(d[k])])
    np.savez_compressed(out, **res)
    print({k: v.shape for k, v in res.items()})


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("collect")
    c.add_argument("--train", type=int, default=3000)
    c.add_argument("--test", type=int, default=1000)
    c.add_argument("--train-start", type=int, default=0, help="first training shape to time (sample prefix is stable)")
    c.add_argument("--test-start", type=int, default=0)
    c.add_argument("--cell-cap", type=float, default=2e8)
    c.add_argument("--budget-s", type=float, default=0.0, help="seconds for the training split, 0 = no limit")
    c.add_argument("--test-budget-s", type=float, default=0.0, help="seconds for the test split, 0 = no limit")
    c.add_argument("--out", default=os.path.join(HERE, "data", "timings.npz"))
    mg = sub.add_parser("merge")
    mg.add_argument("parts", nargs="+")
    mg.add_argument("--out", required=True)
    f = sub.add_parser("fit")
    f.add_argument("db", nargs="?", default=os.path.join(HERE, "data", "timings.npz"))
    f.add_argument("--epochs", type=int, default=3000)
    f.add_argument("--lr", type=float, default=3e-3)
    args = ap.parse_args()
    if args.cmd == "merge":
        merge(args.parts, args.out)
        return
    import torch
    dev = torch.device("cuda:0")
    if args.cmd == "collect":
        train = W.sweep_shapes(args.train, seed=11, cell_cap=args.cell_cap)[args.train_start:]
        test = W.sweep_shapes(args.test, seed=12, cell_cap=args.cell_cap)[args.test_start:]
        out = {}
        for name, shapes in (("train", train), ("test", test)):
            t0 = time.time()
            feats, times, agree = collect(shapes, dev,
                                          budget_s=args.budget_s if name == "train" else args.test_budget_s)
            shapes = shapes[:len(feats)]
            print(f"{name}: {len(shapes)} shapes in {time.time() - t0:.0f} s, all variants bit-exact: "
                  f"{bool(agree.all())}", flush=True)
            out[f"{name}_X"] = feats
            out[f"{name}_ms"] = times
            out[f"{name}_agree"] = agree
            out[f"{name}_shape"] = np.array([[s.m, s.n, s.sigma, int(s.mutated), s.batch, s.seed] for s in shapes],
                                            np.int64)
        os.makedirs(os.path.dirname(args.out), exist_ok=True)
        np.savez_compressed(args.out, variants=np.array([v["name"] for v in CM.VARIANTS]), **out)
    else:
        db = np.load(args.db)
        model, loss = fit(db["train_X"], db["train_ms"], epochs=args.epochs, lr=args.lr)
        rep = report(model, db["test_X"], db["test_ms"])
        rep["train_loss"] = loss
        print(json.dumps(rep, indent=1))
        model.save(extra={"report": rep})


if __name__ == "__main__":
    main()
