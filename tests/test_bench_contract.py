"""The reference arm of bench.py runs on host cores, so its JSON line can be checked here:
one line with the keys the GPU arm prints, the CPU solver's figures in `cpu_baseline` and
`e2e` equal to its own value (host only, no copies)."""
import json
import os
import subprocess
import sys

from conftest import ROOT

KEYS = {"metric", "value", "unit", "impl", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
        "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"}


def run_bench(*args, env=None):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT, capture_output=True,
                       text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    return [ln for ln in r.stdout.splitlines() if ln.strip()]


def test_reference_arm_line():
    lines = run_bench("--impl", "reference", "--steps", "1", "--warmup", "3", "--slice-s", "0.5")
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert KEYS <= set(d)
    assert d["impl"] == "reference" and d["unit"] == "deals/s" and d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 3 and d["n_gpus"] == 1 and d["scaling"] == "weak"
    assert d["config"]["workload"] and d["config"]["jobs_per_deal"] == 5
    cpu = d["cpu_baseline"]
    assert cpu["kind"] in ("reference", "port") and cpu["cores"] >= 1 and cpu["value"] == d["value"] > 0
    assert d["e2e"] == {"value": d["value"], "unit": "deals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_print_nothing():
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    assert run_bench("--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--slice-s", "0.5",
                     env=env) == []
