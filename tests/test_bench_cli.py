"""bench.py's command-line contract on the CPU: the reference arm (the reference estimator
restated in C++, timed on the host) prints one JSON line with the fields the bench line
carries; ranks other than 0 exit without work."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(args, env_extra=None):
    env = dict(os.environ, **(env_extra or {}))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, capture_output=True, text=True,
                       timeout=300, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    return [ln for ln in r.stdout.splitlines() if ln.startswith("{")]


def test_reference_arm_line():
    lines = run_bench(["--impl", "reference", "--steps", "2", "--warmup", "1", "--width", "48", "--height", "27",
                       "--spp", "4"])
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == "Mpaths/s" and d["unit"] == "Mpaths/s"
    assert d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["kind"] in ("port", "reference")
    assert d["e2e"] == {"value": d["value"], "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "random_spheres 48x27" in d["config"]["workload"]


def test_reference_arm_other_ranks_do_no_work():
    lines = run_bench(["--impl", "reference", "--steps", "1", "--warmup", "1", "--width", "48", "--height", "27",
                       "--spp", "4"], {"RANK": "1", "WORLD_SIZE": "2"})
    assert lines == []


def test_reference_arm_config_matches_our_arm():
    """Both arms print the same config dict for the same workload (built by one function)."""
    sys.path.insert(0, ROOT)
    import bench

    lines = run_bench(["--impl", "reference", "--steps", "1", "--warmup", "1", "--width", "48", "--height", "27",
                       "--spp", "4"])
    d = json.loads(lines[0])
    assert set(d["config"]) == {"workload", "width", "height", "spp", "max_depth", "paths_per_step_per_gpu", "l2",
                                "parallelism"}
    assert d["config"]["width"] == 48 and d["config"]["spp"] == 4 and d["config"]["paths_per_step_per_gpu"] == 48 * 27 * 4


def test_cpu_sample_spreads_rows_and_uses_every_thread():
    """The CPU baseline renders a list of rows spread over the frame with OpenMP over the list,
    so all host threads work (one row per call would keep a single thread busy)."""
    sys.path.insert(0, ROOT)
    import bench
    from luminara_b200 import workloads as W

    rows = bench.spread_rows(100, 10, 0.25)
    assert len(set(rows)) == 10 and all(0 <= r < 100 for r in rows)
    more = bench.spread_rows(100, 10, 0.75, exclude=rows)
    assert not set(rows) & set(more)
    world, cfg = W.random_spheres(width=64, height=36, spp=4)
    paths, secs, n_rows, threads = bench.cpu_sample(world, cfg, 0.5, threads=4)
    assert threads == 4 and n_rows >= 8 and paths == n_rows * 64 * 4 and secs > 0
