"""The JSON line contract of bench.py, checked on the reference arm, which
runs the reference's own CPU code (oracle/_ref) on the host cores and so
needs no GPU: one JSON line with the metric, unit and direction of the
headline, its own cpu_baseline and a zero-copy e2e entry."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _ref_built():
    return os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libslcs_ref.so"))


@pytest.mark.skipif(not _ref_built(), reason="oracle/_ref not built")
def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    with open(os.path.join(ROOT, "BASELINE.json")) as f:
        metric = json.load(f)["metric"]
    assert d["impl"] == "reference" and d["metric"] == metric
    assert d["unit"] == "GCUPS" and d["higher_is_better"] is True and d["scaling"] == "weak"
    assert d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["config"]["workload"] == "reads_20000" and d["data"] == "synthetic"
    assert d["value"] > 0 and d["ms_per_step"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["unit"] == d["unit"] and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_gpus_flag_starts_one_rank_per_gpu():
    """--gpus 2 without a torchrun environment starts two ranks of bench.py
    (torch.distributed.run on 127.0.0.1); on a machine without a GPU each
    rank then stops at the device check, so the launcher reports failure."""
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    env["CUDA_VISIBLE_DEVICES"] = ""
    r = subprocess.run([sys.executable, "bench.py", "--gpus", "2", "--steps", "1", "--warmup", "1"], cwd=ROOT,
                       capture_output=True, text=True, timeout=300, env=env)
    out = r.stdout + r.stderr
    # the first rank to stop makes the launcher end the other, so one
    # announcement is certain and the launcher's summary names both ranks
    assert "of 2 (local rank" in out, out[-2000:]
    assert "rank 1 of 2" in out or "local_rank: 1" in out
    assert "rank 0 of 2" in out or "local_rank: 0" in out
    assert "needs a CUDA device" in out
    assert r.returncode != 0


def test_world_size_must_match_gpus():
    env = dict(os.environ, WORLD_SIZE="3", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, "bench.py", "--gpus", "2", "--steps", "1", "--warmup", "1"], cwd=ROOT,
                       capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 2 and "WORLD_SIZE 3" in r.stderr
