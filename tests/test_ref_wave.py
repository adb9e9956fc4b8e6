"""This solver against the reference's own GPU solver on the same deals and the same GPU:
the reference's `dd_gpu` (gpu/gpu_main.cu, its `wave_kernel`, built for sm_100a from its
sources by oracle/build_ref.sh into oracle/_ref/dd_gpu_ref) and this project's `dd_gpu`, both
in their Pgx FILE.npy mode on one file: the first 2,000 deals of the 13-card benchmark set
with the reference CPU solver's tables (tests/golden/k13_bench_2000.npz, written in the
dataset's layout). Each runs a 20 s window (TIME_LIMIT), the reference with its defaults
(WAVE=1, 32,768 threads, TT 2^10) and this solver at 32,768 lanes and on the full grid;
both must check every finished result against the file's tables with none wrong. The
node rates are printed, not asserted: 10,000 jobs fill only part of either solver's lanes,
and in that regime the reference's kernel is the faster one (its 32,768 threads run a
lane each over every SM; this solver's full-load phases are thinly filled)."""
import os
import re
import subprocess

import pytest

from conftest import ROOT, load_golden
import pgx_np

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref", "dd_gpu_ref")
OURS = os.path.join(ROOT, "dds_gpu_b200", "_lib", "dd_gpu")


def run(exe, path, n, env):
    r = subprocess.run([exe, path, "0", str(n), "10"], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, **env))
    out = r.stdout
    m = re.search(r"^GPU: ([0-9.]+)s, [0-9]+ deals/s \([0-9]+ strain-solves/s\), ([0-9]+) nodes/solve$", out, re.M)
    w = re.search(r"^([0-9]+) wrong of ([0-9]+) checked$", out, re.M)
    f = re.search(r"^finished jobs: ([0-9]+) in", out, re.M)
    assert m and w and f, out + r.stderr
    sec, nodes_per_solve = float(m.group(1)), float(m.group(2))
    return {"rc": r.returncode, "wrong": int(w.group(1)), "checked": int(w.group(2)), "jobs": int(f.group(1)),
            "nodes_per_s": nodes_per_solve * n * 5 / sec}


def test_same_deals_as_the_reference_wave_kernel(ddg, tmp_path, capsys):
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref/dd_gpu_ref not built (the reference's sources are not here)")
    g = load_golden("k13_bench_2000.npz")
    n = g["hands"].shape[0]
    path = str(tmp_path / "bench2000.npy")
    pgx_np.write(path, g["hands"], g["tricks"])
    ref = run(REF, path, n, {"WAVE": "1", "THREADS": "32768", "TIME_LIMIT": "20", "CHECK": "0"})
    same = run(OURS, path, n, {"THREADS": "32768", "TIME_LIMIT": "20"})
    full = run(OURS, path, n, {"TIME_LIMIT": "20"})
    with capsys.disabled():
        print(f"\nwave_kernel (32,768 threads): {ref}\nthis solver (32,768 lanes): {same}\n"
              f"this solver (full grid): {full}")
    for r in (ref, same, full):
        assert r["wrong"] == 0 and r["checked"] > 0 and r["rc"] == 0 and r["nodes_per_s"] > 0
