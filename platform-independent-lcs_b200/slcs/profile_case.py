"""Small, self-contained launches for ncu captures.

    python -m slcs.profile_case batch [npairs]     # one batch launch (read/window pairs)
    python -m slcs.profile_case pair  [length]     # one square uniform pair
    python -m slcs.profile_case braid [k] [cutoff] # one staggered product of overlap k
    python -m slcs.profile_case default 131072     # the 131072 mutated pair, default configuration

Each case runs one warm-up launch and then the launch to capture, and checks
the device status word; it holds a few hundred MB on the device at most.
"""
import sys

import numpy as np
import torch

import slcs
from slcs import workloads as W


def main():
    kind = sys.argv[1] if len(sys.argv) > 1 else "batch"
    size = int(sys.argv[2]) if len(sys.argv) > 2 else 0
    tm = int(sys.argv[3]) if len(sys.argv) > 3 else 0
    dev = torch.device("cuda:0")
    if kind == "batch":
        batch = W.reads_20000(npairs=size or 20000)
        _, total = batch.strand_offsets()
        cfg = slcs.Config.make(tile_m=tm or None)
        plan = slcs.BatchPlan(slcs.pair_descs(batch), cfg)
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
        cfg = slcs.Config.make(tile_m=tm or None, wait_ms=600000)  # tm 0: the library's rule
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
        cfg = slcs.Config.make(braid_cutoff=tm or None)
        for _ in range(2):
            slcs.braid_multiply(P, Q, k, False, cfg=cfg)
        torch.cuda.synchronize()
    else:
        raise SystemExit(f"unknown case {kind}")
    slcs.device_status(0)
    print(f"profile case {kind} {size} done")


if __name__ == "__main__":
    main()
