"""Config 5 parity: on a seeded sample of the cost-model sweep's shapes
(every alphabet of {2, 4, 20, 256}, i.i.d. and mutated content, single pairs
and batches of a thousand or more, a side of 2^17 or more), every kernel
variant the cost model can choose -- batch launch plans and single-pair
tilings with each steady-ant cutoff -- must return exactly the strands of
the CPU oracle (Lcs_Semi_Reference2, src/lcs_residual_fixup.hpp:4-70)."""
import numpy as np
import pytest

import oracle as O
from slcs import autotune as AT
from slcs import costmodel as CM
from slcs import workloads as W

pytestmark = pytest.mark.gpu

CELL_LIMIT = 4e7  # per shape, so that the oracle finishes in about a second


def _sample():
    shapes = [s for s in W.sweep_shapes(2000, seed=12, cell_cap=2e8) if s.cells <= CELL_LIMIT]
    pick = []
    for sigma in (2, 4, 20, 256):
        for mutated in (False, True):
            cand = [s for s in shapes if s.sigma == sigma and s.mutated == mutated]
            pick += [c for c in cand if c.batch == 1][:2]
            pick += [c for c in cand if 1 < c.batch <= CM.PAIR_BATCH_MAX][:1]
            pick += [c for c in cand if c.batch > CM.PAIR_BATCH_MAX][:2]
    pick += [s for s in shapes if s.batch >= 1000][:2]
    pick += [s for s in shapes if max(s.m, s.n) >= 1 << 17][:3]
    seen, out = set(), []
    for s in pick:
        if s.seed not in seen:
            seen.add(s.seed)
            out.append(s)
    return out


def test_sample_covers_the_sweep():
    s = _sample()
    assert {x.sigma for x in s} == {2, 4, 20, 256}
    assert {x.mutated for x in s} == {False, True}
    assert any(x.batch == 1 for x in s) and any(x.batch >= 1000 for x in s)
    assert any(max(x.m, x.n) >= 1 << 17 for x in s)
    assert len(s) >= 30


def test_every_variant_matches_the_oracle_on_sweep_shapes(cuda):
    import torch
    import slcs
    checked = 0
    for sh in _sample():
        descs, a, b, total = AT.gpu_shape(sh, cuda)
        ah, bh = a.cpu().numpy(), b.cpu().numpy()
        want = O.comb_batch(ah, bh, descs["a_offset"], descs["b_offset"], descs["m"], descs["n"],
                            descs["out_offset"], total)
        ok = CM.applicable(len(descs))
        for i, v in enumerate(CM.VARIANTS):
            if not ok[i]:
                continue
            plan = None if CM.is_pair(i) else slcs.BatchPlan(descs, CM.variant_config(i, use_graph=False))
            out = torch.full((total,), -7, dtype=torch.int32, device=cuda)
            AT.run_variant(i, descs, a, b, out, plan)
            torch.cuda.synchronize()
            slcs.device_status(0)
            assert np.array_equal(out.cpu().numpy(), want), (v["name"], sh)
            if plan is not None:
                plan.close()
            checked += 1
    assert checked > 300
