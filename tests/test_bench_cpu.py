"""bench.py's CPU side: the reference arm's JSON line (the one line a
benchmark harness parses) and the CPU baseline's timing protocol, on the
small uniform-100k workload."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_contract_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "uniform-100k",
                          "--steps", "2", "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == "Msplats/s sorted (bit-exact stable order)" and d["unit"] == "Msplats/s"
    assert d["higher_is_better"] is True and d["steps"] == 2 and d["warmup"] == 1
    assert d["value"] > 0 and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "Msplats/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"] == "uniform-100k" and d["config"]["splats_per_step"] == 100_000


def test_reference_arm_other_ranks_do_no_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "uniform-100k",
                          "--steps", "1", "--warmup", "0"], cwd=ROOT, capture_output=True, text=True, timeout=600,
                         env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    assert not [ln for ln in out.stdout.splitlines() if ln.startswith("{")]


def test_cpu_baseline_is_the_median_of_five_runs():
    sys.path.insert(0, ROOT)
    import bench
    from winding_b200 import workloads as W
    jobs = [W.uniform_100k(seed=5, n=20_000, cull=0.5), W.uniform_100k(seed=6, n=30_000, cull=0.0)]
    value, sample = bench.cpu_baseline(jobs, 0.5, 1)
    assert value > 0
    assert sample.startswith("median of 5 runs")
    lo, hi = (float(x) for x in sample.split("runs ")[-1].split(" Msplats/s")[0].split("-"))
    assert lo <= value <= hi
