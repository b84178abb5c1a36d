"""The bench's CPU arm keeps its JSON contract: one line with the metric,
value and unit of the GPU arm's line, impl "reference", a cpu_baseline
describing the run and an e2e object with no host copies.  Runs the arm on
the smallest workload (64^3 particles, 128^3 mesh, one step) on the host
cores; no GPU."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(*args):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"),
                          *args], capture_output=True, text=True,
                         timeout=300, cwd=ROOT,
                         env=dict(os.environ, RANK="0", WORLD_SIZE="1"))
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    return json.loads(lines[0])


def test_reference_arm_line():
    d = _run("--impl", "reference", "--config", "config1", "--steps", "1",
             "--warmup", "0")
    assert d["impl"] == "reference"
    assert d["metric"] == "COLA particle-updates/s (64^3 particles, 128^3 mesh)"
    assert d["unit"] == "particle-updates/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0
    assert d["config"]["workload"] == "cola_64p_128m_L64"
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port"
    assert cb["cores"] >= 1 and "no sampling" in cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_of_the_ensemble_is_unavailable():
    d = _run("--impl", "reference", "--config", "config5")
    assert d["impl"] == "reference" and "unavailable" in d
