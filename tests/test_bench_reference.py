"""CPU: the reference arm of bench.py (--impl reference) prints one JSON line
with the keys the bench contract names: the FP64 oracle timed on host cores
over a bounded sample of the workload."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "1", "--cpu-seconds", "1"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "Voigt evals/s"
    assert d["value"] > 0 and d["ms_per_step"] > 0 and d["higher_is_better"] is True
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    # ms_per_step is one whole step (the state's pairs) at the sampled rate;
    # the sample's own wall time is reported apart
    assert cb["state_pairs"] > 1e10
    assert abs(d["ms_per_step"] - 1e3 * cb["state_pairs"] / d["value"]) < 1e-9 * d["ms_per_step"]
    assert 0 < d["sample_s"] < d["ms_per_step"] * 1e-3
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("hitemp")
    # the same workload dict as our arm prints
    sys.path.insert(0, ROOT)
    import bench
    assert d["config"] == json.loads(json.dumps(bench.workload_config(bench.workload("hitemp"))))
