"""Generate the golden fixtures in tests/golden/ from the reference's own code.

Run in a container where the reference sources exist (oracle/Makefile builds
them into oracle/_ref/libslcs_ref.so):

    python tests/golden/make_golden.py            # everything but the 2^20 pair
    python tests/golden/make_golden.py --big      # also the 1048576 x 1048576 pair

Every value below comes from the reference's functions (Lcs_Semi_Reference2,
PermutationMatrix::FromStrands / hash, staggered_multiply), never from the
CUDA engine.  Pairs too large for one host thread are combed as column strips
by the reference procedure and merged with the reference's staggered_multiply
(a composition of reference functions only).
"""
import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "platform-independent-lcs_b200"))

import oracle as O  # noqa: E402
from slcs import workloads as W  # noqa: E402


def ref_hash_pair(a, b, strips=1):
    if strips == 1:
        h, v = O.ref_comb(a, b)
        hv, c2r = O.ref_hash_from_strands(h, v)
        return hv, c2r
    c2r = O.ref_comb_strips(a, b, strips)
    return int(O.ref_lib().ref_hash_col_to_row(c2r.ctypes.data_as(O._i32p), len(c2r))), c2r


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--big", action="store_true")
    args = ap.parse_args()
    if O.ref_lib() is None:
        raise SystemExit("oracle/_ref/libslcs_ref.so is missing: the reference sources are needed")
    path = os.path.join(HERE, "golden.json")
    g = json.load(open(path)) if os.path.exists(path) else {}

    cases = []
    for (m, n, sa, sb) in [(7330, 9944, 888, 999), (9771, 11302, 888, 999), (19771, 24302, 888, 999),
                           (256, 256, 1000, 1001), (4096, 4096, 888, 999)]:
        a, b = O.mt19937_binary(m, sa), O.mt19937_binary(n, sb)
        hv, _ = ref_hash_pair(a, b)
        cases.append({"m": m, "n": n, "seed_a": sa, "seed_b": sb, "hash": hv})
        print("test_default", m, n, hv, flush=True)
    g["test_default"] = cases

    a, b = W.pair_4096()
    hv, c2r = ref_hash_pair(a, b)
    np.save(os.path.join(HERE, "pair_4096_col_to_row.npy"), c2r.astype(np.int32))
    g["pair_4096"] = {"hash": hv, "file": "pair_4096_col_to_row.npy"}
    print("pair_4096", hv, flush=True)

    t = time.time()
    a, b = W.pair_131072_mutated()
    hv, c2r = ref_hash_pair(a, b, strips=64)
    g["pair_131072_mutated"] = {"hash": hv, "sha256_col_to_row": hashlib.sha256(c2r.tobytes()).hexdigest()}
    print("pair_131072_mutated", hv, f"{time.time() - t:.1f}s", flush=True)

    batch = W.reads_20000()
    off, total = batch.strand_offsets()
    ab = batch.a_blob.astype(np.int32)
    bb = batch.b_blob.astype(np.int32)
    out = O.ref_comb_batch(ab, bb, batch.a_off, batch.b_off, batch.ms, batch.ns, off, total)
    g["reads_20000"] = {"npairs": batch.npairs, "cells": batch.cells,
                        "sha256_strands": hashlib.sha256(out.tobytes()).hexdigest()}
    print("reads_20000", g["reads_20000"], flush=True)

    if args.big:
        t = time.time()
        a, b = W.pair_1m()
        hv, c2r = ref_hash_pair(a, b, strips=256)
        g["pair_1M"] = {"hash": hv, "sha256_col_to_row": hashlib.sha256(c2r.tobytes()).hexdigest(),
                        "seconds": round(time.time() - t, 1)}
        print("pair_1M", g["pair_1M"], flush=True)

    with open(path, "w") as f:
        json.dump(g, f, indent=1)


if __name__ == "__main__":
    main()
