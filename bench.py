#!/usr/bin/env python
"""Benchmark of the B200 semi-local LCS engine.

Metric: GCUPS (cell updates per second / 1e9) of the batched, tuned combing
path on the read-versus-window workload (20,000 pairs, lognormal read lengths),
with the plain per-pair launch loop and the 2^20 x 2^20 pair measured beside
it, and the dominant kernel stated against the measured integer roofline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl slcs|reference]
    python bench.py --case batch|pair|default|braid [size] [tile_m|cutoff]

With N > 1 (under torchrun, or launched by bench.py itself when no
WORLD_SIZE is set) one batch of N x 20,000 pairs is dealt out over the ranks
longest first (weak scaling: 20,000 pairs per GPU, no data-path collective);
the time is the maximum over ranks.

--case runs one small, self-contained launch for an ncu capture (one warm-up
launch, then the launch to capture; a few hundred MB on the device at most):
  batch [npairs] [tile_m]   the read/window batch (default 20,000 pairs)
  pair [length] [tile_m]    one square uniform pair (default 65536)
  default [131072|1048576]  the 131072 mutated pair (or the 2^20 pair), default rule
  braid [k] [cutoff]        one staggered product of overlap k (default 2^18)
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "platform-independent-lcs_b200"))

METRIC = "GCUPS on 1 B200: batched+cost-model-tuned vs plain per-pair; % of INT roofline"
UNIT = "GCUPS"
L2_FLUSH_BYTES = 256 << 20


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["slcs", "reference"], default="slcs")
    ap.add_argument("--no-extras", action="store_true", help="skip the per-pair loop and the 2^20 pair")
    ap.add_argument("--case", nargs="+", metavar="ARG", help="one small launch for an ncu capture (see above)")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


# ---------------------------------------------------------------------------
# clocks sampled during the timed region (NVML, read only)
# ---------------------------------------------------------------------------
class ClockSampler:
    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
               0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, device_index: int):
        self.samples, self.reasons = [], set()
        self.ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.max_mhz = None
        self._stop = threading.Event()

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for b, name in self.REASONS.items():
                    if bits & b and b != 0x1:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.001)  # the 20-step timed region lasts about 8 ms

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *exc):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": len(self.samples)}


def read_traffic(kernel_key: str):
    """DRAM bytes per launch recorded from an ncu capture (profiles/*.md)."""
    prof = os.path.join(ROOT, "profiles")
    if not os.path.isdir(prof):
        return None
    for fn in sorted(os.listdir(prof)):
        if not fn.endswith((".md", ".txt")):
            continue
        for line in open(os.path.join(prof, fn)):
            if line.startswith(f"traffic_bytes_per_launch[{kernel_key}]:"):
                try:
                    return float(line.split(":", 1)[1].split()[0])
                except ValueError:
                    return None
    return None


# ---------------------------------------------------------------------------
# reference arm: the reference's own CPU code (oracle/_ref) on host cores
# ---------------------------------------------------------------------------
def run_reference(args, batch):
    """The reference's CPU code over the whole batch per step, all host threads."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    kind = "reference" if O.ref_lib() is not None else "port"
    threads = os.cpu_count() or 1
    off, total = batch.strand_offsets()
    if kind == "reference":
        ab, bb = batch.a_blob.astype(np.int32), batch.b_blob.astype(np.int32)
        step = lambda: O.ref_comb_batch(ab, bb, batch.a_off, batch.b_off, batch.ms, batch.ns, off, total,
                                        nthreads=threads)
    else:
        step = lambda: O.comb_batch(batch.a_blob, batch.b_blob, batch.a_off, batch.b_off, batch.ms, batch.ns,
                                    off, total, nthreads=threads)
    for _ in range(max(1, min(args.warmup, 2))):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    value = batch.cells / dt / 1e9
    desc = f"all {batch.npairs} read/window pairs ({batch.cells} cells) per step"
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "reads_20000", "pairs": batch.npairs},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def cpu_baseline(batch):
    """The reference's CPU code timed on this host's cores on the whole batch."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    threads = os.cpu_count() or 1
    off, total = batch.strand_offsets()
    if O.ref_lib() is not None:
        ab, bb = batch.a_blob.astype(np.int32), batch.b_blob.astype(np.int32)
        t0 = time.perf_counter()
        out = O.ref_comb_batch(ab, bb, batch.a_off, batch.b_off, batch.ms, batch.ns, off, total, nthreads=threads)
        dt = time.perf_counter() - t0
        kind = "reference"
    else:
        t0 = time.perf_counter()
        out = O.comb_batch(batch.a_blob, batch.b_blob, batch.a_off, batch.b_off, batch.ms, batch.ns, off, total,
                           nthreads=threads)
        dt = time.perf_counter() - t0
        kind = "port"
    return {"value": batch.cells / dt / 1e9, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"all {batch.npairs} pairs ({batch.cells} cells), one pass, {dt:.2f} s"}, out


def relaunch_ranks(args) -> int:
    """--gpus N > 1 without a torchrun environment: start N ranks of this
    script under torch.distributed.run (one process per GPU) and return the
    launcher's exit status."""
    import socket
    import subprocess
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.run(cmd).returncode


def run_case(case) -> int:
    """One small launch for an ncu capture: a warm-up launch, then the launch
    to capture, and a check of the device status word."""
    import torch
    import slcs
    from slcs import workloads as W
    kind = case[0]
    size = int(case[1]) if len(case) > 1 else 0
    knob = int(case[2]) if len(case) > 2 else 0
    dev = torch.device("cuda:0")
    if kind == "batch":
        batch = W.reads_20000(npairs=size or 20000)
        _, total = batch.strand_offsets()
        plan = slcs.BatchPlan(slcs.pair_descs(batch), slcs.Config.make(tile_m=knob or None))
        a = torch.from_numpy(batch.a_blob).to(dev)
        b = torch.from_numpy(batch.b_blob).to(dev)
        out = torch.empty(total, dtype=torch.int32, device=dev)
        for _ in range(2):
            plan.run(a, b, out)
        torch.cuda.synchronize()
        plan.close()
    elif kind == "pair":
        n = size or 65536
        rng = np.random.default_rng(1)
        a = torch.from_numpy(rng.integers(0, 4, n, dtype=np.uint8)).to(dev)
        b = torch.from_numpy(rng.integers(0, 4, n, dtype=np.uint8)).to(dev)
        out = torch.empty(2 * n, dtype=torch.int32, device=dev)
        cfg = slcs.Config.make(tile_m=knob or None, wait_ms=600000)  # tile 0: the library's rule
        for _ in range(2):
            slcs.comb_pair(a, b, cfg=cfg, out=out)
        torch.cuda.synchronize()
    elif kind == "default":
        a_h, b_h = W.pair_131072_mutated() if (size or 131072) == 131072 else W.pair_1m()
        a = torch.from_numpy(a_h).to(dev)
        b = torch.from_numpy(b_h).to(dev)
        out = torch.empty(len(a_h) + len(b_h), dtype=torch.int32, device=dev)
        for _ in range(2):
            slcs.comb_pair(a, b, cfg=slcs.Config.make(wait_ms=600000), out=out)
        torch.cuda.synchronize()
    elif kind == "braid":
        k = size or (1 << 18)
        rng = np.random.default_rng(2)
        P = torch.from_numpy(rng.permutation(k + 1000).astype(np.int32)).to(dev)
        Q = torch.from_numpy(rng.permutation(k + 3000).astype(np.int32)).to(dev)
        cfg = slcs.Config.make(braid_cutoff=knob or None)
        for _ in range(2):
            slcs.braid_multiply(P, Q, k, False, cfg=cfg)
        torch.cuda.synchronize()
    else:
        print(f"unknown case {kind}", file=sys.stderr)
        return 2
    slcs.device_status(0)
    print(f"case {' '.join(case)} done")
    return 0


def main():
    args = parse_args()
    rank, world, local = dist_env()
    if args.case:
        return run_case(args.case)
    from slcs import workloads as W
    if args.impl == "reference":
        if rank != 0:
            return 0
        batch = W.reads_20000()
        print(json.dumps(run_reference(args, batch)), flush=True)
        return 0
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        return relaunch_ranks(args)
    if world != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but WORLD_SIZE {world}", file=sys.stderr)
        return 2

    import torch
    import slcs
    from slcs import distributed as D
    from slcs import tuning

    if world > 1:
        print(f"bench.py: rank {rank} of {world} (local rank {local})", file=sys.stderr, flush=True)
    if not torch.cuda.is_available():
        print("bench.py: the GPU arm needs a CUDA device", file=sys.stderr)
        return 2
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist

    # One batch of 20,000 pairs per GPU, dealt out longest first (rank 0 of a
    # single GPU gets the whole 20,000-pair batch, whose digest is committed).
    full = W.reads_20000(npairs=20000 * world)
    if world > 1:
        shard = D.shard_pairs(full.ms.astype(np.int64) * full.ns, world)[rank]
        batch = full.subset(shard)
    else:
        batch = full
    descs = slcs.pair_descs(batch)
    _, total = batch.strand_offsets()
    a_d = torch.from_numpy(batch.a_blob).to(dev)
    b_d = torch.from_numpy(batch.b_blob).to(dev)
    out = torch.empty(total, dtype=torch.int32, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream()

    def time_config(c, reps=3):
        """Best of `reps` runs of one variant on this batch (before the timed region)."""
        p = slcs.BatchPlan(descs, c)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p.run(a_d, b_d, out)
        best = float("inf")
        for _ in range(reps):
            flush.zero_()
            e0.record(stream)
            p.run(a_d, b_d, out)
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        p.close()
        return best

    cfg, tuned_by, tuning_info = tuning.choose_batch_config(batch, timer=time_config)
    plan = slcs.BatchPlan(descs, cfg)

    int_ops, cell_rate = slcs.probe_int_rates()
    roof_gcups = int_ops / 5.0 / 1e9

    for _ in range(args.warmup):
        plan.run(a_d, b_d, out)
        flush.zero_()
    torch.cuda.synchronize()
    slcs.device_status(local)

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    with sampler:
        for e0, e1 in ev:
            flush.zero_()
            e0.record(stream)
            plan.run(a_d, b_d, out)
            e1.record(stream)
        torch.cuda.synchronize()
    if pg:
        pg.barrier()
    slcs.device_status(local)
    step_ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    total_ms = float(sum(step_ms))
    if pg:
        t = torch.tensor([total_ms], dtype=torch.float64, device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    cells_all = full.cells
    value = cells_all / (ms_per_step * 1e-3) / 1e9
    kern_gcups = batch.cells / (ms_per_step * 1e-3) / 1e9

    # parity of the timed output with the committed golden digest (one GPU:
    # the batch is exactly the 20,000 pairs whose strands were digested)
    bitexact = None
    if world == 1:
        import hashlib
        g = json.load(open(os.path.join(ROOT, "tests", "golden", "golden.json")))
        bitexact = hashlib.sha256(out.cpu().numpy().tobytes()).hexdigest() == g["reads_20000"]["sha256_strands"]

    # end to end: host buffers through the C ABI, copies inside the timed
    # region.  The strands come back as int16 (every id of these pairs is
    # below 2^15, so the values are exactly the int32 ones; checked below),
    # and, beside it, as int32.
    a_h = torch.from_numpy(batch.a_blob).pin_memory().numpy()
    b_h = torch.from_numpy(batch.b_blob).pin_memory().numpy()
    o_h = torch.empty(total, dtype=torch.int32).pin_memory().numpy()
    o16_h = torch.empty(total, dtype=torch.int16).pin_memory().numpy()
    e2e_steps = max(3, min(args.steps, 50))

    def e2e_time(run, o):
        for _ in range(2):
            run(a_h, b_h, o)
        if pg:
            pg.barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            run(a_h, b_h, o)
        dt = (time.perf_counter() - t0) / e2e_steps
        if pg:
            t = torch.tensor([dt], dtype=torch.float64, device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            dt = float(t.item())
        return dt

    e2e32_s = e2e_time(plan.run_host, o_h)
    e2e_s = e2e_time(plan.run_host16, o16_h)
    same16 = bool(np.array_equal(o16_h.astype(np.int32), o_h))
    e2e = {"value": cells_all / e2e_s / 1e9, "unit": UNIT, "h2d_bytes_per_step": int(a_h.nbytes + b_h.nbytes),
           "d2h_bytes_per_step": int(o16_h.nbytes), "ms_per_step": e2e_s * 1e3,
           "strands": "int16 (slcs_batch_plan_run_host16)", "int16_equals_int32_strands": same16,
           "int32": {"value": cells_all / e2e32_s / 1e9, "ms_per_step": e2e32_s * 1e3,
                     "d2h_bytes_per_step": int(o_h.nbytes), "strands": "int32 (slcs_batch_plan_run_host)"}}

    extras = {}
    if not args.no_extras and rank == 0:
        extras = tuning.secondary_measurements(batch, a_d, b_d, out, roof_gcups, dev,
                                               sampler=lambda: ClockSampler(local))

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": "reads_20000", "pairs_per_gpu": batch.npairs, "pairs": full.npairs,
                   "cells_per_gpu_step": batch.cells,
                   "variant": dict(plan.info, graph=bool(cfg.use_graph)),
                   "tuned_by": tuned_by, "tuning": tuning_info, "l2": "flushed between steps (256 MiB write)",
                   "parallelism": f"{world} shards of one batch, dealt longest first (weak)"},
        "e2e": e2e,
        "gpu_launches": args.steps * plan.launches,
        "roofline": {"bound": "int32", "achieved": kern_gcups, "peak": roof_gcups, "unit": "GCUPS",
                     "frac": kern_gcups / roof_gcups, "traffic": read_traffic("reads_20000"),
                     "peak_source": "measured here: INT32 min/max issue rate / 5 ops per cell",
                     "int32_tops": int_ops / 1e12, "cell_rule_ceiling_gcups": cell_rate / 1e9},
        "clocks": sampler.summary(),
        "bitexact_vs_reference": bitexact,
    }
    line.update(extras)
    if rank == 0 and world == 1:
        cb, ref_out = cpu_baseline(batch)
        line["cpu_baseline"] = cb
    if rank == 0:
        print(json.dumps(line), flush=True)
    del plan
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
