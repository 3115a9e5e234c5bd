"""The reference arm of bench.py on the CPU: one JSON line with the contract's keys, timed on the
oracle port over a small workload (the GPU arm is exercised on the GPU box)."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_prints_one_contract_line(tmp_path):
    env = dict(os.environ, TMPDIR=str(tmp_path))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "t0",
                        "--steps", "2", "--warmup", "3"], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "s/timestep" and d["higher_is_better"] is False
    assert d["steps"] == 2 and d["warmup"] == 3 and d["value"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "s/timestep", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["pcg_iters_per_step"] > 0
