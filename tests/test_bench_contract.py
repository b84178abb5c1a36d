"""The bench's CPU arm keeps its JSON contract: one line with the metric,
value and unit of the GPU arm's line, impl "reference", a cpu_baseline
describing the run and an e2e object with no host copies.  Runs the arm on
the smallest workload (64^3 particles, 128^3 mesh, one step) on the host
cores; and the clock record that goes beside every GPU line reads the
throttle reasons from nvidia-smi's output.  No GPU."""
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


def test_clock_summary_reads_throttle_reasons():
    # nvidia-smi --query-gpu=<ClockSampler.FIELDS> --format=csv,noheader,
    # nounits lines: index, sm, max sm, power, active mask, then the four
    # reasons the timing rules name
    sys.path.insert(0, ROOT)
    import bench
    lines = [
        "0, 1965, 1965, 700.1, 0x0000000000000000, Not Active, Not Active, "
        "Not Active, Not Active",
        "0, 1890, 1965, 1001.3, 0x0000000000000004, Not Active, Not Active, "
        "Not Active, Active",
        "0, 1900, 1965, 998.0, 0x0000000000000004, Not Active, Not Active, "
        "Not Active, Active",
        "garbage",
        "0, [N/A], 1965, 1.0, 0x0, Not Active, Not Active, Not Active, "
        "Not Active",
    ]
    s = bench.ClockSampler.summarise(lines)
    assert s["samples"] == 3 and s["sm_mhz"] == 1900.0
    assert s["sm_max_mhz"] == 1965.0 and s["reasons"] == ["sw_power_cap"]
    hot = ["0, 1500, 1965, 900, 0x48, Active, Not Active, Active, Not Active"]
    assert bench.ClockSampler.summarise(hot)["reasons"] == [
        "hw_slowdown", "sw_thermal_slowdown"]
    assert bench.ClockSampler.summarise([])["sm_mhz"] is None


def test_reference_arm_under_torchrun_prints_once():
    # launched as the multi-GPU runs are (one process per rank): rank 0 runs
    # the CPU arm and prints its line, the other rank exits 0 without work
    out = subprocess.run(
        [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
         "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
         "--master-port", "29531", os.path.join(ROOT, "bench.py"),
         "--impl", "reference", "--config", "config1", "--steps", "1",
         "--warmup", "0"],
        capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0
