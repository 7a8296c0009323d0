"""bench.py's reference arm on the host cores (no GPU): one JSON line with the contract's keys.

`bench.py --impl reference` times the reference coretrace built from its sources
(oracle/_ref/coretrace_ref.so) on every host core, on the same metric, unit and workload
as the B200 arm; without that library it prints an `unavailable` line and exits 0.  Run here
on a small field and a 2-second sample so the CPU suite stays short.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0",
           "--cpu-seconds", "2", "--hits", "20000", "--helios", "120"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" in d:
        assert not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "coretrace_ref.so"))
        return
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "scaling", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 1
    assert d["unit"] == "ray-stage intersections/s"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["heliostats"] == 120 and d["config"]["hits_per_step_per_gpu"] == 20000


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun only rank 0 times the reference; the other ranks print nothing and exit 0."""
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
           "--warmup", "0", "--cpu-seconds", "2", "--hits", "20000", "--helios", "120"]
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    assert not [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
