"""The benchmark's JSON contract on the CPU: the reference arm's line (a tiny functional-preset case
of the CPU prover), the workload naming shared by both arms, and the helpers that summarise
latencies and sampled clocks."""
import argparse
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_reference_arm_line_keeps_the_contract():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "1", "--log-n", "6", "--width", "8", "--preset", "functional"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "impl", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 1
    assert line["unit"] == "proofs/s" and line["higher_is_better"] is True and line["value"] > 0
    assert line["metric"] == bench.METRIC
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["unit"] == "proofs/s"
    assert line["e2e"] == {"value": line["value"], "unit": "proofs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == "wide-Fibonacci 2^6x8, functional preset"


def test_both_arms_name_the_same_workload():
    args = argparse.Namespace(log_n=20, width=100, preset="secure", in_flight=8)
    ours, ref = bench.config_block(args, 8), bench.config_block(args)
    assert ours["workload"] == ref["workload"] == "wide-Fibonacci 2^20x100, secure preset"
    assert ours["proofs_per_step"] == 8 and ref["proofs_per_step"] == 1
    assert "larger than L2" in ours["l2"]


def test_percentiles():
    xs = [5.0, 1.0, 3.0, 2.0, 4.0]
    assert bench.pct(xs, 50) == 3.0
    assert bench.pct(xs, 0) == 1.0 and bench.pct(xs, 100) == 5.0
    assert abs(bench.pct(xs, 99) - 4.96) < 1e-9
    assert bench.pct([], 50) is None


def test_clock_summary_reports_throttle_reasons():
    s = bench.ClockSampler(0)
    s.lines = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
               "0, 1900, 1965, 990.5, 0x4, Not Active, Not Active, Not Active, Active",
               "0, 1965, 1965, 710.0, 0x0, Not Active, Not Active, Not Active, Not Active",
               "garbage"]
    summ = s.summary()
    assert summ["sm_mhz"] == 1965.0 and summ["sm_max_mhz"] == 1965.0 and summ["samples"] == 3
    assert summ["reasons"] == ["sw_power_cap"]
    assert bench.ClockSampler(0).summary()["reasons"] == ["nvidia-smi unavailable"]
