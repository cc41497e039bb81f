"""The output contract of bench.py's reference arm (CPU): `--impl reference` times the
reference's own evaluate_cpu_omp, compiled from its sources, on the host cores and
prints exactly one JSON line carrying the metric, the CPU baseline that it is and an
end-to-end figure with no host<->device bytes."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_json_line(ref_mod):
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "config", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["value"] > 0 and d["unit"] == "evals/s" and d["higher_is_better"] is True
    assert d["config"]["workload"] == "L300_N5000"
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    # the same workload keys as the GPU arm's config, nothing about the implementation
    assert {"ncol", "nrow", "planted_pairs", "seed", "parallelism"} <= set(d["config"])
    assert "path" not in d["config"]
