"""bench.py's reference arm runs on the host alone (no GPU) and prints the contract's JSON line."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_prints_its_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "synaptic events/s"
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["higher_is_better"] is True
    # the line names the sample it times and counts the bench steps it timed
    assert line["steps"] == 1 and line["warmup"] == 3
    assert "50,000-neuron" in line["config"]["workload"] and line["config"]["timed_sim_steps"] == 90
    assert line["cpu_baseline"]["value"] == line["value"]


def test_profile_steps_refuses_multi_rank_launches():
    """--profile-steps prints per-step events for an ncu capture of one GPU; under torchrun
    (WORLD_SIZE > 1) it stops before touching a device."""
    env = dict(os.environ, WORLD_SIZE="2", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--profile-steps", "3"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert r.returncode != 0
    assert "--profile-steps profiles one GPU" in r.stderr
