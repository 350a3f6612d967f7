"""bench.py's reference arm on the CPU: the JSON line it prints keeps the
benchmark contract (the same metric, unit and direction as the CUDA arm, the
reference arm's impl tag, a cpu_baseline describing the run and an e2e
object with no host/device copies), and the arm never maps the engine
library into its process (its pairs come from the oracle's generator)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, capture_output=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr.decode()[-3000:]
    lines = [ln for ln in r.stdout.decode().splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout.decode()[-2000:]
    return json.loads(lines[0])


def test_reference_arm_line():
    d = _run("--impl", "reference", "--workload", "c1", "--steps", "2", "--warmup", "1")
    assert d["impl"] == "reference"
    assert d["unit"] == "GCUPS" and d["higher_is_better"] is True
    assert d["metric"].startswith("GCUPS & pairs/s on 1 B200")
    assert d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0 and d["pairs_per_s"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert d["config"]["workload"].startswith("c1:")
    # the arm exits non-zero when /proc/self/maps shows the engine library,
    # so the zero exit status checked by _run covers that
