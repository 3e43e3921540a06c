"""bench.py's reference arm runs on the host alone; its JSON line carries the
keys the measurement contract names (the GPU arm is exercised on a B200)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "c1", "--steps", "1",
                        "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["n_gpus"] == 1 and d["steps"] == 1
    assert d["metric"] == "input Mfaces/s" and d["unit"] == "Mfaces/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"] and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # one step's time is the measured sample; the whole-workload estimate is labelled
    ex = d["extrapolated"]
    assert abs(ex["measured_s_per_step"] * 1e3 - d["ms_per_step"]) < 1e-6 * d["ms_per_step"]
    assert ex["estimated_s_whole_workload"] > 0 and "basis" in ex
    # no GPU here: the reference's own GPU build is reported as unavailable
    assert d["reference_gpu_stage2"] is None or "unavailable" in d["reference_gpu_stage2"]
