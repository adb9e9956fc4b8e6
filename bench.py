#!/usr/bin/env python
"""Benchmark: exact double-dummy deals/s on B200s (one process per GPU, weak scaling).

Workload: seeded uniformly random 13-card deals (seed 2; deals [0, 20,000) are the
20,000-deal benchmark set, and the solve runs on over deals [0, SET_SIZE) of the same
stream so that every lane holds a job through the whole run), all 5 strains x 4 declarers,
one job per (deal, strain) with the four declarers sharing a TT of 2^10 buckets per lane,
inputs resident in HBM; rank r takes deals [SET_SIZE r, SET_SIZE (r+1)). The set is solved as one
resumable solve (ddg_solve_begin); a step is one slice of it (ddg_solve_continue,
--slice-s seconds, every lane's search state kept in HBM between slices): one kernel launch,
timed with CUDA events on its stream.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --profile-case [--lanes L] [--set-size D]   # one slice to capture under ncu

value: exact deals/s in steady state. The GPU searches exactly the reference's nodes job
for job (same bounds, move order and TT decisions; the tests check it node for node), so a
deal costs the GPU the reference's search nodes, and with every lane busy the rate at
which whole tables complete is the node rate divided by the mean nodes per deal of the
workload (the renewal-reward rate of a solver that always has the next job). The mean is
measured, not assumed: tests/golden/k13_bench_2000.npz holds the reference's complete
tables and per-job node counts for deals [0, 2,000) of the set (the learned guide's
searches: tests/golden/k13_bench_2000_guided.npz, from the host replay of this solver's
stage machine with the guide's seeds and leads). `value` is the guided solver's (the guide
seeds the search and orders the root leads; the searches decide every answer), `plain`
the same measurement without the guide. `finished_deals_per_s` is the reference README's
window metric (jobs finished in the timed slices / 5 / time), which favours the easy
deals and is reported beside it, for both arms.
e2e: the same through the host API with, every step, the deals copied in from pinned host
memory and all results copied out. roofline: TT bytes of the launch (64 per probe, 16 per
entry read, 80 per store) per second of kernel time, against the measured HBM copy
bandwidth. cpu_baseline / --impl reference: the reference's own CPU solver
(dd_solve_strain from its src/dd.h, compiled into oracle/_ref/cpu_window, which also makes
the deals itself) on every host core over the same slices. parity: every job of deals
[0, 2,000) that a run finished against the reference's tables, and every job the GPU and
the CPU run both finished against each other. same_deals (N = 1): the reference's own GPU
solver (its wave_kernel, gpu/gpu_main.cu built for sm_100a into oracle/_ref/dd_gpu_ref, in
the reference arm's line) and this solver (its dd_gpu, in this arm's line) each run a
--wave-s window on one Pgx file of deals [0, 2,000), checked against its tables.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "exact DD deals/s on 1 B200, learned-guided vs plain; nodes/deal; p99 ms"
SET_SEED, SET_K = 2, 13
SET_SIZE = 60000  # deals per GPU: far more jobs than the lanes finish in a run, so no lane idles
BENCH_SET = 20000
JPD = 5
SAMPLE = os.path.join(ROOT, "tests", "golden", "k13_bench_2000.npz")
GUIDED_SAMPLE = os.path.join(ROOT, "tests", "golden", "k13_bench_2000_guided.npz")
# DRAM bytes (read + write) per search node of one launch of this workload's own shape
# (TT 2^10, 75,776 lanes, third 0.5 s slice), from `bench.py --profile-case --warmup 2
# --slice-s 0.5` under ncu (dram__bytes_read.sum + dram__bytes_write.sum = 27.04 + 10.04
# GB over 350.2 M nodes).
DRAM_BYTES_PER_NODE = 105.9
WORKLOAD = ("13-card seeded random deals, all 5 strains x 4 declarers, exact TT 2^10 buckets per lane, "
            "one job per (deal, strain)")


def parse(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--slice-s", type=float, default=2.0, help="seconds per step (one slice of the solve)")
    p.add_argument("--tt-log2", type=int, default=10)
    p.add_argument("--lanes", type=int, default=0, help="0 = fill the GPU")
    p.add_argument("--block", type=int, default=0, help="threads (lanes) per block; 0 = library default (512)")
    p.add_argument("--min-blocks", type=int, default=0)
    p.add_argument("--schedule", type=int, default=0, help="0 block-phase kernel, 1 queue kernel")
    p.add_argument("--flat-moves", type=int, default=0,
                   help="0 (default) / 1: lead-move weights spread over the block; -1: per-lane loop")
    p.add_argument("--free-below", type=int, default=0, help="the solver's free_below (0 = its default)")
    p.add_argument("--free-pack", type=int, default=0, help="the solver's free_pack (0 = its default)")
    p.add_argument("--set-size", type=int, default=SET_SIZE)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-guide", action="store_true", help="plain solver only (no learned guide)")
    p.add_argument("--wave-s", type=float, default=10.0,
                   help="seconds per run of the same-deals comparison with the reference's GPU solver (0 = skip)")
    p.add_argument("--profile-case", action="store_true",
                   help="warm-up slices then one slice, nothing else (the launch to capture under ncu)")
    return p.parse_args(argv)


def launch_plan(gpus, env):
    """What to do with --gpus N: 'run' (this process is one of the N ranks, or N = 1),
    'spawn' (start N ranks under torch.distributed.run), or 'refuse' (started as a rank of
    a job of another size)."""
    world = env.get("WORLD_SIZE")
    if world is None:
        return "spawn" if gpus > 1 else "run"
    return "run" if int(world) == gpus else "refuse"


def spawn_ranks(gpus, argv):
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + argv
    return subprocess.call(cmd)


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def deal_set(rank, size=SET_SIZE):
    from dds_gpu_b200 import make_deals
    return make_deals(SET_SEED, rank * size, size, SET_K)


def sample_costs():
    """Mean search nodes per deal of the workload: the reference's complete solves of deals
    [0, 2,000) (plain), and the guided search's (host replay with the guide's seeds and
    leads), with the standard error of each mean; None where the file is missing."""
    import numpy as np
    out = {}
    for key, path in (("plain", SAMPLE), ("guided", GUIDED_SAMPLE)):
        if not os.path.exists(path):
            out[key] = None
            continue
        with np.load(path) as z:
            per_deal = z["nodes_jpd5"].astype(np.float64).reshape(-1, 5).sum(axis=1)
            meta = {k: z[k] for k in z.files if k in ("params_sum",)}
        out[key] = {"nodes_per_deal": float(per_deal.mean()), "deals": int(per_deal.size),
                    "stderr": float(per_deal.std(ddof=1) / np.sqrt(per_deal.size)), **{k: float(v) for k, v in meta.items()}}
    return out


def sample_tables():
    import numpy as np
    with np.load(SAMPLE) as z:
        return z["tricks"].reshape(-1, 20)


def parity_against(got, want):
    """Entries of `got` (n, 20) that are solved (not 255) in the rows both hold, compared."""
    m = min(len(got), len(want))
    g, w = got[:m], want[:m]
    done = (g != 255) & (w != 255)
    return int(done.sum()), bool((g[done] == w[done]).all())


# ---- CPU reference path (baseline only) -------------------------------------------------

def cpu_window(a, size, slices, tables_out=None):
    """The reference's CPU solver over deals [0, size) of the set for `slices` slices of
    a.slice_s (oracle/_ref/cpu_window, built from the reference's sources; else the C
    restatement's oracle/_build/cpu_window). It makes the deals itself."""
    exe = os.path.join(ROOT, "oracle", "_ref", "cpu_window")
    if not os.path.exists(exe):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
        exe = os.path.join(ROOT, "oracle", "_build", "cpu_window")
    args = [exe, f"gen:{SET_SEED}:{size}:{SET_K}", str(a.tt_log2), str(host_cores()), str(a.slice_s), str(slices),
            str(a.warmup)]
    if tables_out:
        args.append(tables_out)
    out = subprocess.run(args, check=True, capture_output=True, text=True, timeout=a.slice_s * slices + 120).stdout
    return json.loads(out.strip().splitlines()[-1])


def cpu_measure(a, costs, size=BENCH_SET):
    import numpy as np
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "tables.bin")
        r = cpu_window(a, size, a.warmup + a.steps, path)
        tables = np.fromfile(path, dtype=np.uint8).reshape(-1, 20)
    t = a.steps * a.slice_s
    t_jobs = sum(r["jobs"][a.warmup:])
    t_nodes = sum(r["nodes"][a.warmup:])
    nps = t_nodes / t
    plain = costs.get("plain")
    value = nps / plain["nodes_per_deal"] if plain else t_jobs / JPD / t
    sample = (f"deals [0, {size}) of seed {SET_SEED} solved in order by {r['threads']} threads, one TT each; "
              f"slices {a.warmup}..{a.warmup + a.steps - 1} of {a.slice_s:g} s timed (first {a.warmup} = warm-up): "
              f"{t_nodes} nodes, {t_jobs} jobs finished; value = nodes/s / reference nodes per deal")
    return {"value": value, "unit": "deals/s", "cores": r["threads"], "kind": r["kind"], "sample": sample,
            "nodes_per_s": nps, "finished_deals_per_s": t_jobs / JPD / t,
            "job_ms": {"p50": r["job_ms_p50"], "p99": r["job_ms_p99"]}}, tables


def run_dd_gpu(exe, path, n, env, timeout=300):
    """One `dd_gpu FILE.npy 0 n 10` run (the reference's gpu/gpu_main.cu driver or this
    project's, same argv and output lines): every finished result is checked against the
    file's tables; returns rc, wrong/checked, finished jobs and the node rate."""
    import re
    try:
        r = subprocess.run([exe, path, "0", str(n), "10"], capture_output=True, text=True, timeout=timeout,
                           env=dict(os.environ, **env))
    except (OSError, subprocess.TimeoutExpired) as e:
        return {"rc": None, "error": f"{type(e).__name__}: {e}"[-400:]}
    out = r.stdout
    m = re.search(r"^GPU: ([0-9.]+)s, [0-9]+ deals/s \([0-9]+ strain-solves/s\), ([0-9]+) nodes/solve$", out, re.M)
    w = re.search(r"^([0-9]+) wrong of ([0-9]+) checked$", out, re.M)
    f = re.search(r"^finished jobs: ([0-9]+) in", out, re.M)
    if not (m and w and f):
        return {"rc": r.returncode, "error": (out + r.stderr)[-400:]}
    sec, nodes_per_solve = float(m.group(1)), float(m.group(2))
    return {"rc": r.returncode, "wrong": int(w.group(1)), "checked": int(w.group(2)), "jobs": int(f.group(1)),
            "seconds": sec, "nodes_per_s": nodes_per_solve * n * JPD / sec}


def same_deals(a, exe, runs):
    """The reference's GPU solver (`wave_kernel`) and this one on one Pgx file: deals
    [0, 2,000) of the benchmark set with the reference CPU solver's tables, a.wave_s
    seconds each (TIME_LIMIT). `runs` maps a name to the driver's environment."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import pgx_np
    if not (os.path.exists(exe) and os.path.exists(SAMPLE)):
        return {"unavailable": f"{os.path.relpath(exe, ROOT)} or the 2,000-deal fixture is missing"}
    with np.load(SAMPLE) as z:
        hands, tricks = z["hands"], z["tricks"]
    out = {"deals": f"deals [0, {len(hands)}) of the benchmark set in the Pgx .npy layout, checked against "
                    "the reference CPU solver's tables",
           "tt_log2": 10, "window_s": a.wave_s}
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "bench2000.npy")
        pgx_np.write(path, hands, tricks)
        for name, env in runs.items():
            out[name] = run_dd_gpu(exe, path, len(hands), dict(env, TIME_LIMIT=f"{a.wave_s:g}"),
                                   timeout=a.wave_s + 240)
    return out


def config_dict(a, world):
    return {"workload": WORKLOAD,
            "deal_set": (f"seed {SET_SEED}, K={SET_K}; deals [0, {BENCH_SET}) are the benchmark set, the solve runs "
                         f"over [0, {a.set_size}) per GPU so no lane idles"),
            "tt_log2": a.tt_log2, "jobs_per_deal": JPD, "step": f"one {a.slice_s:g} s slice of the resumable solve",
            "parallelism": f"dp{world} (own deal range per GPU, no collective on the data path)",
            "l2": "flushed between steps (256 MiB write); the TT working set (GBs) is far above L2"}


def reference_arm(a, rank, world):
    if rank != 0:
        return
    costs = sample_costs()
    cpu, tables = cpu_measure(a, costs)
    n, eq = parity_against(tables, sample_tables()) if costs.get("plain") else (0, True)
    line = {"metric": METRIC, "value": cpu["value"], "unit": "deals/s", "impl": "reference", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * a.slice_s,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic", "config": config_dict(a, world),
            "nodes_per_s": cpu["nodes_per_s"], "finished_deals_per_s": cpu["finished_deals_per_s"],
            "job_ms": cpu["job_ms"], "nodes_per_deal": costs.get("plain"),
            "parity": {"checked": n, "equal": eq, "against": "reference tables of deals [0, 2000) (fixture)"},
            "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cpu["value"], "unit": "deals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if a.wave_s > 0 and world == 1:
        line["same_deals"] = same_deals(a, os.path.join(ROOT, "oracle", "_ref", "dd_gpu_ref"), {
            "reference_wave_kernel_32768_threads": {"WAVE": "1", "THREADS": "32768", "CHECK": "0"}})
    print(json.dumps(line), flush=True)


# ---- GPU arm -----------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for row in self.f.read().strip().splitlines():
            c = [x.strip() for x in row.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                mx.append(float(c[2]))
            except ValueError:
                continue
            for name, v in zip(names, c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def combine_ranks(world, dev, elapsed_ms, e2e_ms, jobs, e2e_jobs, nodes):
    """Whole-job figures: the slowest rank's times (max) and every rank's work (sum). The
    only collectives of the bench; the solves themselves exchange nothing."""
    if world <= 1:
        return elapsed_ms, e2e_ms, jobs, e2e_jobs, nodes
    import torch
    t = torch.tensor([elapsed_ms, e2e_ms or 0.0], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    c = torch.tensor([jobs, e2e_jobs, nodes], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(c)
    return t[0].item(), (t[1].item() if e2e_ms else None), c[0].item(), c[1].item(), c[2].item()


def quantiles_ms(start, end, warm_end):
    """p50 / p99 search time (ms) of the jobs finished in the timed slices (finished now,
    not yet at the end of the warm-up)."""
    import numpy as np
    done = (end > 0) & (warm_end == 0) & (start > 0)
    if not done.any():
        return {"p50": None, "p99": None, "jobs": 0}
    d = np.sort((end[done] - start[done]).astype(np.float64) / 1e6)
    return {"p50": float(d[len(d) // 2]), "p99": float(d[min(len(d) - 1, int(0.99 * len(d)))]), "jobs": int(len(d))}


def our_arm(a, rank, world, local_rank):
    import numpy as np
    import torch
    import dds_gpu_b200 as ddg
    import dds_gpu_b200.guide as ddg_guide

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    deals = deal_set(rank, a.set_size)
    solver = ddg.Solver(tt_log2=a.tt_log2, lanes=a.lanes, block=a.block, jobs_per_deal=JPD, device=local_rank,
                        min_blocks=a.min_blocks, schedule=a.schedule, flat_moves=a.flat_moves,
                        free_below=a.free_below, free_pack=a.free_pack)
    n = deals.shape[0]
    host_in = torch.from_numpy(deals.view(np.int64)).pin_memory()
    dev_in = host_in.to(dev)
    dev_out = torch.empty((n, 20), dtype=torch.uint8, device=dev)
    d_end = torch.zeros(n * JPD, dtype=torch.int64, device=dev)
    d_start = torch.zeros(n * JPD, dtype=torch.int64, device=dev)
    solver.set_job_times(d_end.data_ptr(), d_start.data_ptr())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    cs = stream.cuda_stream

    if a.profile_case:  # the launch to capture: W warm-up slices, then one slice
        solver.begin(dev_in.data_ptr(), n, dev_out.data_ptr(), stream=cs)
        for _ in range(a.warmup):
            solver.resume(a.slice_s, stream=cs)
        _, st = solver.resume(a.slice_s, stream=cs)
        torch.cuda.synchronize(dev)
        if rank == 0:
            print(json.dumps({"profile_case": True, "launches": a.warmup + 1, "last_launch": {
                k: st[k] for k in ("nodes", "tt_probes", "tt_entry_reads", "tt_stores", "tt_bytes", "kernel_ms",
                                   "lanes", "grid", "block", "jobs_done", "enter_exit", "phase_warps", "phase_items",
                                   "phase_cycles", "free_rounds", "free_cycles", "iterations")}}), flush=True)
        solver.close()
        return

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def window(d_seed=0, d_hint=0):
        """W warm-up and K timed slices of one resumable solve of the set."""
        solver.begin(dev_in.data_ptr(), n, dev_out.data_ptr(), d_seeds=d_seed, d_hints=d_hint, stream=cs)
        for _ in range(a.warmup):  # warm-up slices (untimed)
            flush.zero_()
            solver.resume(a.slice_s, stream=cs)
        torch.cuda.synchronize(dev)
        warm_end = d_end.cpu().numpy()
        sampler = ClockSampler(local_rank)
        stats = []
        barrier()
        torch.cuda.synchronize(dev)
        sampler.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.steps):
            flush.zero_()
            stats.append(solver.resume(a.slice_s, stream=cs)[1])
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        clocks = sampler.stop()
        start, end = d_start.cpu().numpy(), d_end.cpu().numpy()
        return {"stats": stats, "ms": e0.elapsed_time(e1), "clocks": clocks, "tables": dev_out.cpu().numpy(),
                "lat": quantiles_ms(start, end, warm_end), "started_all": bool((start > 0).all())}

    # The learned guide (when its trained weights are there): NS seeds and root leads for
    # the whole set, computed on the GPU before the solve.
    d_seed = d_hint = None
    guide_info = None
    params = None if a.no_guide else ddg_guide.load_weights()
    if params is not None:
        guide = ddg.Guide(device=local_rank, max_rows=8192, params=params)
        d_seed = torch.empty(n * 20, dtype=torch.int8, device=dev)
        d_hint = torch.empty(n * 20, dtype=torch.int8, device=dev)
        torch.cuda.synchronize(dev)
        g0 = time.perf_counter()
        guide.predict(dev_in.data_ptr(), n, d_seed.data_ptr(), d_hint.data_ptr())
        torch.cuda.synchronize(dev)
        guide_info = {"predict_ms": 1e3 * (time.perf_counter() - g0), "rows": n * 20,
                      "params_sum": float(params.astype(np.float64).sum())}
        guide.close()

    costs = sample_costs()
    plain_run = window()
    runs = {"plain": plain_run}
    if d_seed is not None:
        runs["guided"] = window(d_seed.data_ptr(), d_hint.data_ptr())
        seeds = d_seed.cpu().numpy().reshape(n, 5, 4).astype(int)
        t = runs["guided"]["tables"].reshape(n, 5, 4).astype(int)
        ns = np.where(np.arange(4) % 2 == 0, t, 13 - t)
        done = t <= 13
        guide_info.update({"seed_exact": float((seeds == ns)[done].mean()) if done.any() else None,
                           "seed_within_one": float((abs(seeds - ns) <= 1)[done].mean()) if done.any() else None})
    # the guide's nodes per deal belong to these weights only
    g_cost = costs.get("guided")
    guided_cost_ok = bool(guide_info and g_cost and abs(g_cost.get("params_sum", 0) - guide_info["params_sum"]) < 1e-3)

    # End to end through the host API: each step copies the deals in from pinned host memory,
    # runs the slice and copies every result out.
    e2e_ms, e2e_nodes, e2e_jobs = None, 0, 0
    if not a.no_e2e:
        host_out = torch.empty((n, 20), dtype=torch.uint8).pin_memory()
        solver.begin(dev_in.data_ptr(), n, dev_out.data_ptr(), stream=cs,
                     d_seeds=d_seed.data_ptr() if d_seed is not None else 0,
                     d_hints=d_hint.data_ptr() if d_hint is not None else 0)
        for _ in range(a.warmup):
            solver.resume(a.slice_s, hands_host=host_in.data_ptr(), out_host=host_out.data_ptr(), stream=cs)
        barrier()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(a.steps):
            flush.zero_()
            st = solver.resume(a.slice_s, hands_host=host_in.data_ptr(), out_host=host_out.data_ptr(), stream=cs)[1]
            e2e_nodes += st["nodes"]
            e2e_jobs += st["jobs_done"]
        torch.cuda.synchronize(dev)
        e2e_ms = 1e3 * (time.perf_counter() - t0)
        barrier()

    head = "guided" if ("guided" in runs and guided_cost_ok) else "plain"
    summary = {}
    for key, run in runs.items():
        nodes = sum(st["nodes"] for st in run["stats"])
        jobs = sum(st["jobs_done"] for st in run["stats"])
        ms, _, jobs_all, _, nodes_all = combine_ranks(world, dev, run["ms"], None, jobs, 0, nodes)
        cost = costs.get(key)
        if key == "guided" and not guided_cost_ok:
            cost = None
        nps = nodes_all / (ms * 1e-3)
        summary[key] = {"value": nps / cost["nodes_per_deal"] if cost else None, "unit": "deals/s",
                        "nodes_per_s": nps, "nodes_per_deal": cost,
                        "finished_deals_per_s": jobs_all / JPD / (ms * 1e-3), "jobs_finished": int(jobs_all),
                        "nodes_per_s_by_step": [st["nodes"] / (st["kernel_ms"] * 1e-3) for st in run["stats"]],
                        "job_ms": run["lat"], "queue_ran_dry": run["started_all"], "ms": ms}
    e2e_ms_all, _, e2e_nodes_all, _, _ = combine_ranks(world, dev, e2e_ms or 0.0, None, e2e_nodes, 0, 0)

    cpu = cpu_tables = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cpu, cpu_tables = cpu_measure(a, costs)

    if rank != 0:
        solver.close()
        return
    # parity: the reference's tables of deals [0, 2000) and the CPU run's finished jobs
    checked, equal = 0, True
    against = []
    if os.path.exists(SAMPLE):
        want = sample_tables()
        for run in runs.values():
            c, e = parity_against(run["tables"], want)
            checked, equal = checked + c, equal and e
        against.append("reference tables of deals [0, 2000) (fixture made by the reference's solver)")
    if cpu_tables is not None:
        for run in runs.values():
            c, e = parity_against(run["tables"], cpu_tables)
            checked, equal = checked + c, equal and e
        against.append("the reference CPU solver's tables of this run")
    both = (runs["plain"]["tables"] != 255)
    if "guided" in runs:
        both &= runs["guided"]["tables"] != 255
        guided_equal_plain = bool((runs["plain"]["tables"][both] == runs["guided"]["tables"][both]).all())
    else:
        guided_equal_plain = None

    run = runs[head]
    stats = run["stats"]
    kernel_ms = sum(st["kernel_ms"] for st in stats)
    alg_bytes = sum(64 * st["tt_probes"] + 16 * st["tt_entry_reads"] + 80 * st["tt_stores"] for st in stats)
    counted = sum(st["tt_bytes"] for st in stats)
    nodes = sum(st["nodes"] for st in stats)
    it = [sum(st["phase_warps"][k] for st in stats) for k in range(5)]
    ln = [sum(st["phase_items"][k] for st in stats) for k in range(5)]
    peak, peak_kind = peaks()
    launches = len(stats)
    achieved = (alg_bytes / launches) / (kernel_ms / launches * 1e-3) / 1e9 if kernel_ms else 0.0
    eff = {name: (ln[k] / (32.0 * it[k]) if it[k] else None)
           for k, name in enumerate(["cheap", "enter_lead", "enter_follow", "moves_lead", "moves_follow"])}
    s_head = summary[head]
    value = s_head["value"] if s_head["value"] is not None else s_head["finished_deals_per_s"]
    elapsed_ms = s_head["ms"]
    line = {
        "metric": METRIC, "value": value, "unit": "deals/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": elapsed_ms / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": config_dict(a, world),
        "value_is": (f"{head} solver: nodes/s over the timed slices / the workload's mean nodes per deal"
                     if s_head["value"] is not None else "finished jobs / 5 / s (no node-cost sample)"),
        "tuning": {"lanes": stats[0]["lanes"] if stats else 0, "block": stats[0]["block"] if stats else a.block,
                   "schedule": a.schedule, "flat_moves": a.flat_moves,
                   "free_below": a.free_below, "free_pack": a.free_pack,
                   "guide": ("learned guide: NS seeds (stepping search) + root leads" if head == "guided"
                             else "off (plain DDS move order)")},
        "nodes_per_s": s_head["nodes_per_s"], "nodes_per_deal": s_head["nodes_per_deal"],
        "finished_deals_per_s": s_head["finished_deals_per_s"], "job_ms": s_head["job_ms"],
        "guided": summary.get("guided"), "plain": summary["plain"],
        "guide": guide_info, "guided_tables_equal_plain": guided_equal_plain,
        "parity": {"checked": checked, "equal": equal, "against": against},
        "warp_efficiency": eff,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": (DRAM_BYTES_PER_NODE * nodes / launches) if DRAM_BYTES_PER_NODE else None,
                     "kernel": f"ddg::batch_kernel<{solver.block_shape}>",
                     "algorithmic_bytes": (f"64 B per TT probe + 16 B per entry read + 80 B per store: "
                                           f"{alg_bytes / max(1, nodes):.1f} B/node (the kernel's own count, which "
                                           f"also charges each store its tag-line read: "
                                           f"{counted / max(1, nodes):.1f} B/node)")},
        "clocks": run["clocks"],
        "gpu_launches": launches,
    }
    if e2e_ms:
        e2e_cost = costs.get(head) if (head == "plain" or guided_cost_ok) else None
        e2e_val = (e2e_nodes_all / (e2e_ms_all * 1e-3) / e2e_cost["nodes_per_deal"]) if e2e_cost else None
        line["e2e"] = {"value": e2e_val if e2e_val is not None else e2e_jobs / JPD / (e2e_ms * 1e-3),
                       "unit": "deals/s", "h2d_bytes_per_step": n * 32, "d2h_bytes_per_step": n * 20}
    if cpu:
        line["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        line["cpu_baseline"].update({"nodes_per_s": cpu["nodes_per_s"],
                                     "finished_deals_per_s": cpu["finished_deals_per_s"], "job_ms": cpu["job_ms"]})
        line["vs_cpu_nodes_per_s"] = s_head["nodes_per_s"] / cpu["nodes_per_s"] if cpu["nodes_per_s"] else None
    solver.close()
    if a.wave_s > 0 and world == 1:
        exe = os.path.join(ROOT, "dds_gpu_b200", "_lib", "dd_gpu")
        line["same_deals"] = same_deals(a, exe, {"32768_lanes": {"THREADS": "32768"}, "full_grid": {}})
    print(json.dumps(line), flush=True)


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    a = parse(argv)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    plan = launch_plan(a.gpus, os.environ)
    if plan == "refuse":
        print(f"bench.py: --gpus {a.gpus} but started as one of {world} ranks", file=sys.stderr)
        return 2
    if plan == "spawn":
        return spawn_ranks(a.gpus, argv)
    if a.impl == "reference":
        reference_arm(a, rank, world)
        return 0
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        our_arm(a, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
