"""The C++ mirror of the reference interface end to end: bin/slcs_test reads a
script in the reference's format, runs registered B200 procedures through
LcsAlgorithmRegistry / SemiLocalLcsImpl, and writes the reference's CSV with
PermutationMatrix::hash, which must equal the reference's golden hashes."""
import csv
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "platform-independent-lcs_b200", "bin", "slcs_test")


def test_script_runner_matches_golden_hashes(tmp_path):
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        cases = json.load(f)["test_default"]
    algos = ["b200", "b200_2_4", "b200_14_8", "b200_16_8", "b200_strips_4_1024", "b200_strips_8_64", "b200_bands_4_256"]
    lines = []
    for alg in algos:
        for c in cases:
            lines.append(f"algorithm={alg} device_type=gpu size_a={c['m']} size_b={c['n']} "
                         f"seed_a={c['seed_a']} seed_b={c['seed_b']}")
    script = tmp_path / "script.txt"
    script.write_text("# B200 procedures on the reference's test cases\n" + "\n".join(lines) + "\n")
    out = tmp_path / "out.csv"
    r = subprocess.run([BIN, str(script), str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    rows = list(csv.DictReader(open(out)))
    assert len(rows) == len(algos) * len(cases)
    want = {(c["m"], c["n"], c["seed_a"], c["seed_b"]): c["hash"] for c in cases}
    for row, line in zip(rows, lines):
        kv = dict(w.split("=") for w in line.split())
        key = (int(kv["size_a"]), int(kv["size_b"]), int(kv["seed_a"]), int(kv["seed_b"]))
        assert int(row["hash"]) == want[key], (row["algorithm"], key)
