"""bench.py's reference arm on the host (CPU only): the JSON line the bench contract asks
for, with the reference's own CPU search (check.cpp's brute force, compiled from the
reference sources into oracle/_ref) as the measured implementation."""
import json
import os
import subprocess
import sys

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
        "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
        "cpu_baseline", "e2e")


def test_reference_arm_prints_the_contract_line():
    env = {**os.environ, "CUDA_VISIBLE_DEVICES": ""}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--scale", "0.002", "--steps", "1", "--warmup", "1",
                        "--cpu-seconds", "1"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    assert all(k in d for k in KEYS), sorted(set(KEYS) - set(d))
    assert d["impl"] == "reference" and d["metric"] == "queries/s" and d["unit"] == "queries/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["config"]["workload"] == "knn_multicloud_4096" and d["config"]["k"] == 32
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"]
    assert cb["kind"] == ("reference" if oracle.ref_available() else "port")
    assert d["e2e"] == {"value": d["value"], "unit": "queries/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
