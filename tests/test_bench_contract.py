"""bench.py's contract pieces that need no GPU: the reference arm's JSON line (it runs on
host cores and loads nothing of the product), its rank handling, and what --gpus N does
in each launch situation."""
import json
import os
import subprocess
import sys

from conftest import ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402

KEYS = {"metric", "value", "unit", "impl", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
        "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e", "parity", "nodes_per_s"}


def run_bench(*args, env=None):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, capture_output=True,
                       text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    return [ln for ln in r.stdout.splitlines() if ln.strip()]


def test_reference_arm_line():
    lines = run_bench("--impl", "reference", "--steps", "2", "--warmup", "2", "--slice-s", "1", "--wave-s", "0")
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert KEYS <= set(d)
    assert d["impl"] == "reference" and d["unit"] == "deals/s" and d["higher_is_better"] is True
    assert d["steps"] == 2 and d["warmup"] == 2 and d["n_gpus"] == 1 and d["scaling"] == "weak"
    assert d["config"] == bench.config_dict(bench.parse(["--slice-s", "1"]), 1)  # the GPU arm's config
    cpu = d["cpu_baseline"]
    assert cpu["kind"] in ("reference", "port") and cpu["cores"] >= 1 and cpu["value"] == d["value"] > 0
    assert d["e2e"] == {"value": d["value"], "unit": "deals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # value = the CPU's node rate over the workload's mean nodes per deal
    assert abs(d["value"] - d["nodes_per_s"] / d["nodes_per_deal"]["nodes_per_deal"]) < 1e-9 * d["value"]
    assert d["parity"]["equal"] is True and d["parity"]["checked"] > 0
    assert "same_deals" not in d  # the GPU comparison is skipped with --wave-s 0


def test_reference_arm_loads_nothing_of_the_product():
    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '1', "
            "'--slice-s', '0.5', '--wave-s', '0']; import bench; bench.main(sys.argv[1:]); "
            "maps = open('/proc/self/maps').read(); print(json.dumps({'ddg': 'libddg' in maps}))")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert json.loads(r.stdout.strip().splitlines()[-1]) == {"ddg": False}


def test_reference_arm_other_ranks_print_nothing():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    assert run_bench("--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--slice-s", "0.5",
                     env=env) == []


def test_gpus_launch_plan():
    assert bench.launch_plan(1, {}) == "run"
    assert bench.launch_plan(4, {}) == "spawn"            # starts its own 4 ranks
    assert bench.launch_plan(4, {"WORLD_SIZE": "4"}) == "run"
    assert bench.launch_plan(8, {"WORLD_SIZE": "2"}) == "refuse"
    assert bench.launch_plan(1, {"WORLD_SIZE": "1"}) == "run"


def test_gpus_mismatch_is_refused():
    env = dict(os.environ, RANK="0", LOCAL_RANK="0", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "4"], cwd=ROOT,
                       capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 2 and "--gpus 4" in r.stderr


def test_dd_gpu_output_parsing(tmp_path):
    """same_deals reads the reference's `dd_gpu` output lines (gpu/gpu_main.cu:277,307,340);
    a stand-in printing them is parsed into the node rate, the check and the finished jobs,
    and a run without them is reported as an error, not a number."""
    fake = tmp_path / "dd_gpu"
    fake.write_text("#!/bin/sh\n"
                    "echo '10048 threads, 2000 deals, 10000 solves, TT 320 KB/solve, 3.29 GB total'\n"
                    "echo 'finished jobs: 2873 in 10.1 s = 56.8 full-job deals/s'\n"
                    "echo 'GPU: 10.11s, 198 deals/s (989 strain-solves/s), 117550 nodes/solve'\n"
                    "echo '0 wrong of 14132 checked'\n")
    fake.chmod(0o755)
    r = bench.run_dd_gpu(str(fake), "unused.npy", 2000, {})
    assert r["rc"] == 0 and r["wrong"] == 0 and r["checked"] == 14132 and r["jobs"] == 2873
    assert abs(r["nodes_per_s"] - 117550 * 2000 * 5 / 10.11) < 1e-6 * r["nodes_per_s"]
    broken = tmp_path / "broken"
    broken.write_text("#!/bin/sh\necho 'no device'\nexit 1\n")
    broken.chmod(0o755)
    r = bench.run_dd_gpu(str(broken), "unused.npy", 2000, {})
    assert r["rc"] == 1 and "error" in r and "nodes_per_s" not in r
    slow = tmp_path / "slow"
    slow.write_text("#!/bin/sh\nsleep 30\n")
    slow.chmod(0o755)
    r = bench.run_dd_gpu(str(slow), "unused.npy", 2000, {}, timeout=1)
    assert r["rc"] is None and "TimeoutExpired" in r["error"]
