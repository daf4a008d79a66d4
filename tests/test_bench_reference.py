"""bench.py --impl reference on the CPU: the reference arm runs the oracle
port of the serial reference step, one instance per host core (capped
here), and prints the contract's JSON line."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_its_line():
    env = dict(os.environ, SPHG_HOST_CORES="2")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                          "--warmup", "1"], capture_output=True, text=True, env=env, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] == 2
    assert line["unit"] == "particle-steps/s" and line["higher_is_better"] is True
    assert line["cpu_baseline"]["cores"] == 2
    # the same config as the arm on the GPU
    assert line["config"]["workload"] == "two_phase_912k" and line["config"]["particles"] == 912016
    assert line["cpu_baseline"]["kind"] == "port"
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
