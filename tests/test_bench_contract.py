"""bench.py's reference arm runs on the CPU alone (it times the reference's
torch CPU path): one tiny run of it, checked for the JSON line the driver
reads (metric, value, unit, impl, config, cpu_baseline, e2e)."""
import json
import os
import subprocess
import sys

from conftest import ROOT


def test_reference_arm_prints_the_contract_line():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "c0",
                        "--steps", "1", "--warmup", "3", "--ref-batch", "2"],
                       capture_output=True, text=True, cwd=ROOT, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference" and line["unit"] == "patterns/s" and line["value"] > 0
    assert line["metric"] and line["config"]["workload"].startswith("c0")
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
