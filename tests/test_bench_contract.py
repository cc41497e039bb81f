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


def test_tensor_peak_follows_the_held_clock():
    """The roofline's bf16 denominator is the measured peak taken at the clock nearer
    the one the timed region held: burst near the maximum clock, sustained near the
    power-capped clock; the region's length decides only without clock samples."""
    sys.path.insert(0, ROOT)
    import bench
    peaks = {"bf16_tflops": 1672.5, "bf16_tflops_sustained": 1395.1, "sm_max_mhz": 1965.0,
             "clocks_under_load": {"sm_mhz_median": 1342.0}}
    peak, name, why = bench.tensor_peak(peaks, "measured", {"sm_mhz": 1882.0}, 1004.0)
    assert (peak, name) == (1672.5, "bf16_tflops") and "1882" in why
    peak, name, _ = bench.tensor_peak(peaks, "measured", {"sm_mhz": 1500.0}, 10.0)
    assert (peak, name) == (1395.1, "bf16_tflops_sustained")
    assert bench.tensor_peak(peaks, "measured", None, 20.0)[1] == "bf16_tflops"
    assert bench.tensor_peak(peaks, "measured", None, 2000.0)[1] == "bf16_tflops_sustained"
    fb = bench.tensor_peak({"bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0},
                           "fallback", {"sm_mhz": 1965.0}, 5.0)
    assert fb[0] == 1590.0 and "absent" in fb[2]
