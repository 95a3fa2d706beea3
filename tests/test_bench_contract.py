"""bench.py's reference arm (the CPU restatement timed on the host cores)
prints the one JSON line of the benchmark contract, and ranks other than 0
exit without work. Runs on CPU at a small size."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SMALL = ["--steps", "1", "--warmup", "3", "--nodes", "512", "--width", "160", "--height", "120", "--gn", "1",
         "--pcg", "2", "--batch", "2"]


def run_bench(extra_env=None):
    env = dict(os.environ)
    env.update(extra_env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", *SMALL],
                          cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)


def test_reference_arm_prints_contract_line():
    p = run_bench()
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    r = json.loads(lines[0])
    assert r["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config"):
        assert key in r, key
    assert r["value"] > 0 and r["unit"] == "solves/s" and r["higher_is_better"] is True
    assert r["steps"] == 1 and r["warmup"] == 3 and r["scaling"] == "weak"
    assert "workload" in r["config"] and r["config"]["nodes"] == 512
    cb = r["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == r["value"] and cb["sample"]
    e2e = r["e2e"]
    assert e2e["value"] == r["value"] and e2e["unit"] == r["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_without_output():
    p = run_bench({"RANK": "1", "WORLD_SIZE": "2"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert not [ln for ln in p.stdout.splitlines() if ln.startswith("{")]


def test_committed_spmv_profile_parses():
    """The headline line's roofline.traffic comes from the committed ncu
    summary; its DRAM row must parse to the read + write bytes."""
    import argparse
    sys.path.insert(0, ROOT)
    import bench
    a = argparse.Namespace(batch=16, nodes=4096, width=640, height=480, precision="mixed", mode="materialized")
    traffic, src = bench.measured_traffic(a)
    assert src is not None and 1e7 < traffic < 1e9


def test_committed_profiles_give_the_summed_dram_bytes():
    """The SpMV summary's row is "R + W MB" for the 16-instance launch; the
    matrix-free summary has one DRAM figure per kernel for 8 instances, which
    the bench sums and scales to its batch."""
    import argparse
    sys.path.insert(0, ROOT)
    import bench
    a = argparse.Namespace(batch=16, nodes=4096, width=640, height=480, precision="mixed", mode="materialized")
    assert bench.measured_traffic(a)[0] == int((110.2 + 2.39) * 1e6)
    a.mode = "matrix_free"
    traffic, src = bench.measured_traffic(a)
    assert src.endswith("apply_pair_matrix_free_torso_3view_4096nodes_8inst.md")
    assert traffic == int((130 + 165) * 1e6 * 2)
    a.batch = 8
    assert bench.measured_traffic(a)[0] is None  # only the headline batch size
