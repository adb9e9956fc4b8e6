#!/usr/bin/env python
"""Benchmark: exact double-dummy deals/s on B200s (one process per GPU, weak scaling).

Workload: the 13-card benchmark set (20,000 seeded uniformly random deals, seed 2,
ddg_make_deals), full 5x4 trick tables, exact TT with 2^10 buckets per lane. One step =
one batch solve of `--batch` consecutive deals of the set (rank r of N takes its own
batch: step s uses deals from ((s*N + r) * batch) mod 20000), inputs already in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Rank 0 prints one JSON line. `value` = deals solved by all ranks / max over ranks of the
device time of the K timed steps (CUDA events on the solve stream, barrier and synchronize
on both sides; L2 flushed between steps). `e2e` = the same metric through the host API
(ddg_solve_batch: pinned host deals in, H2D, solve, D2H of the 20-byte results).
`roofline` = TT bytes the search moved (counted in-kernel) per second of kernel time,
against the measured HBM copy bandwidth. `cpu_baseline` = the reference's own CPU solver
(compiled from its sources into oracle/_ref, else the oracle port) on a bounded sample,
all host cores. `--impl reference` times that CPU path alone as the reference arm.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "exact DD deals/s on 1 B200, learned-guided vs plain; nodes/deal; p99 ms"
SET_SEED, SET_SIZE, SET_K = 2, 20000, 13
WORKLOAD = "13-card seeded random deals, full 5x4 tables, exact TT 2^10 buckets/lane"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--batch", type=int, default=1024, help="deals per step per GPU")
    p.add_argument("--tt-log2", type=int, default=10)
    p.add_argument("--lanes", type=int, default=0, help="0 = fill the GPU")
    p.add_argument("--jpd", type=int, default=20, help="jobs per deal: 5 (per strain) or 20 (per lead)")
    p.add_argument("--block", type=int, default=256)
    p.add_argument("--min-blocks", type=int, default=2)
    p.add_argument("--help-lanes", type=int, default=1, help="1: idle lanes help busy ones (same tricks)")
    p.add_argument("--safety-s", type=float, default=900.0, help="per-step stop; a stopped step is an error")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--cpu-deals", type=int, default=0, help="deals per CPU sample (0 = one per core)")
    return p.parse_args()


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---- CPU reference path (checker/baseline only) ----------------------------------------

def cpu_solver():
    """The reference's CPU solver: oracle/_ref (reference sources) if built, else the port."""
    P = ctypes.c_void_p
    ref = os.path.join(ROOT, "oracle", "_ref", "libddref.so")
    if os.path.exists(ref):
        lib = ctypes.CDLL(ref)
        lib.ref_solve_batch.argtypes = [P, ctypes.c_long, ctypes.c_int, ctypes.c_int, P, P]

        def run(h, tt, threads, out, nodes):
            return lib.ref_solve_batch(h.ctypes.data, h.shape[0], tt, threads, out.ctypes.data, nodes.ctypes.data)
        return run, "reference"
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_build", "libddoracle.so"))
    lib.ddo_solve_batch.restype = ctypes.c_longlong
    lib.ddo_solve_batch.argtypes = [P, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P]

    def run(h, tt, threads, out, nodes):
        r = lib.ddo_solve_batch(h.ctypes.data, h.shape[0], tt, threads, 5, None, out.ctypes.data, nodes.ctypes.data)
        return 0 if r >= 0 else -1
    return run, "port"


def cpu_sample(deals, first, n, tt_log2, threads):
    """Solves deals [first, first+n) of the set on the CPU; returns (seconds, nodes, tables)."""
    import numpy as np
    run, kind = cpu_solver()
    idx = [(first + i) % SET_SIZE for i in range(n)]
    h = np.ascontiguousarray(deals[idx])
    out = np.zeros(n * 20, np.int32)
    nodes = np.zeros(n * 5, np.uint64)
    t0 = time.perf_counter()
    rc = run(h, tt_log2, threads, out, nodes)
    dt = time.perf_counter() - t0
    if rc != 0:
        raise RuntimeError("CPU solver failed")
    return dt, int(nodes.sum()), out.reshape(n, 5, 4), kind


def config_dict(a, world, extra=None):
    d = {"workload": WORKLOAD, "deal_set": f"seed {SET_SEED}, {SET_SIZE} deals, K={SET_K}",
         "deals_per_step_per_gpu": a.batch, "tt_log2": a.tt_log2, "jobs_per_deal": a.jpd,
         "parallelism": f"dp{world} (independent deals per GPU, no collective on the data path)",
         "l2": "flushed between steps (256 MiB write); TT working set is also far above L2"}
    if extra:
        d.update(extra)
    return d


def reference_arm(a, rank, world):
    if rank != 0:
        return
    import numpy as np
    from dds_gpu_b200 import make_deals
    deals = make_deals(SET_SEED, 0, SET_SIZE, SET_K)
    cores = host_cores()
    n = a.cpu_deals or max(4, cores)
    times, nodes = [], 0
    kind = "reference"
    for s in range(a.warmup + a.steps):
        dt, nd, _, kind = cpu_sample(deals, s * n, n, a.tt_log2, cores)
        if s >= a.warmup:
            times.append(dt)
            nodes += nd
    total = sum(times)
    value = a.steps * n / total
    sample = f"{n} deals per step x {a.steps} steps (deals 0..{(a.warmup + a.steps) * n - 1}; first {a.warmup * n} as warm-up), all 20 results"
    line = {"metric": METRIC, "value": value, "unit": "deals/s", "impl": "reference", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * total / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic", "config": config_dict(a, world, {"deals_per_step_per_gpu": n}),
            "nodes_per_deal": nodes / (a.steps * n),
            "cpu_baseline": {"value": value, "unit": "deals/s", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "deals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
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


def our_arm(a, rank, world, local_rank):
    import numpy as np
    import torch
    import dds_gpu_b200 as ddg

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    deals = ddg.make_deals(SET_SEED, 0, SET_SIZE, SET_K)
    solver = ddg.Solver(tt_log2=a.tt_log2, lanes=a.lanes, block=a.block, jobs_per_deal=a.jpd, device=local_rank,
                        min_blocks=a.min_blocks, help=a.help_lanes, time_limit_s=a.safety_s)
    B = a.batch
    nsteps = a.warmup + a.steps

    def step_idx(s):
        start = ((s * world + rank) * B) % SET_SIZE
        return [(start + i) % SET_SIZE for i in range(B)]

    host_in = [torch.from_numpy(np.ascontiguousarray(deals[step_idx(s)]).view(np.int64)).pin_memory()
               for s in range(nsteps)]
    dev_in = [h.to(dev) for h in host_in]
    dev_outs = [torch.empty((B, 20), dtype=torch.uint8, device=dev) for _ in range(nsteps)]
    dev_out = dev_outs[0]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # Warm-up steps (untimed).
    for s in range(a.warmup):
        flush.zero_()
        solver.solve_device(dev_in[s].data_ptr(), B, dev_out.data_ptr(), stream=stream.cuda_stream)
    torch.cuda.synchronize(dev)

    sampler = ClockSampler(local_rank)
    stats = []
    barrier()
    torch.cuda.synchronize(dev)
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for s in range(a.warmup, nsteps):
        flush.zero_()
        stats.append(solver.solve_device(dev_in[s].data_ptr(), B, dev_outs[s].data_ptr(), stream=stream.cuda_stream))
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    clocks = sampler.stop()
    elapsed_ms = e0.elapsed_time(e1)
    # Every result of every timed step must be there (the safety stop leaves 255s).
    unsolved = sum(int((dev_outs[s] == 255).sum().item()) for s in range(a.warmup, nsteps))
    tables = [dev_outs[s].cpu().numpy() for s in range(a.warmup, nsteps)]

    # End to end through the host API: pinned deals in, results out, every step.
    e2e_ms = None
    if not a.no_e2e:
        host_out = torch.empty((B, 20), dtype=torch.uint8).pin_memory()
        lib = ddg.load_library()
        st = ddg._Stats()
        for s in range(a.warmup):
            ddg._check(lib.ddg_solve_batch(solver._h, host_in[s].data_ptr(), B, host_out.data_ptr(), ctypes.byref(st)))
        barrier()
        torch.cuda.synchronize(dev)
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        legacy = torch.cuda.default_stream(dev)
        h0.record(legacy)
        t0 = time.perf_counter()
        for s in range(a.warmup, nsteps):
            flush.zero_()
            ddg._check(lib.ddg_solve_batch(solver._h, host_in[s].data_ptr(), B, host_out.data_ptr(), ctypes.byref(st)))
            assert int(host_out[0, 0]) <= 13
        h1.record(legacy)
        torch.cuda.synchronize(dev)
        wall_ms = 1e3 * (time.perf_counter() - t0)
        e2e_ms = max(h0.elapsed_time(h1), wall_ms)
        barrier()

    if world > 1:
        t = torch.tensor([elapsed_ms, e2e_ms or 0.0], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        elapsed_ms, e2e_ms = t[0].item(), (t[1].item() if e2e_ms else None)

    kernel_ms = sum(s["kernel_ms"] for s in stats)
    nodes = sum(s["nodes"] for s in stats)
    tt_bytes = sum(s["tt_bytes"] for s in stats)
    it = [sum(s["phase_warps"][k] for s in stats) for k in range(5)]
    ln = [sum(s["phase_items"][k] for s in stats) for k in range(5)]
    tasks = sum(s["tasks"] for s in stats)
    if world > 1:
        t = torch.tensor([nodes, tt_bytes], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t)
        nodes_all = t[0].item()
    else:
        nodes_all = nodes

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cores = host_cores()
        n = a.cpu_deals or max(4, cores)
        dt, cn, tables, kind = cpu_sample(deals, 0, n, a.tt_log2, cores)
        cpu = {"value": n / dt, "unit": "deals/s", "cores": cores, "kind": kind,
               "sample": f"deals 0..{n - 1} of the set (5 strains x 4 declarers each), {cores} threads, "
                         f"TT 2^{a.tt_log2} buckets per thread, {dt:.1f} s, {cn / n:.0f} nodes/deal"}
        # The GPU answers for the same deals must match the CPU reference's.
        gpu_tab = solver.solve(deals[:n])
        cpu["tables_equal_gpu"] = bool((gpu_tab == tables).all())

    if rank != 0:
        solver.close()
        return
    peak, peak_kind = peaks()
    achieved = tt_bytes / (kernel_ms * 1e-3) / 1e9 if kernel_ms else 0.0
    deals_total = a.steps * B * world
    value = deals_total / (elapsed_ms * 1e-3)
    eff = {name: (ln[k] / (32.0 * it[k]) if it[k] else None)
           for k, name in enumerate(["cheap", "enter_lead", "enter_follow", "moves_lead", "moves_follow"])}
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        try:
            with open(tfile) as f:
                tj = json.load(f)
            traffic = tj.get("dram_bytes_per_node", 0) * nodes / max(1, len(stats))
        except (OSError, ValueError):
            traffic = None
    line = {
        "metric": METRIC, "value": value, "unit": "deals/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": elapsed_ms / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": config_dict(a, world, {"lanes": stats[0]["lanes"] if stats else 0,
                                         "block": a.block, "guide": "off (plain DDS move order)"}),
        "nodes_per_deal": nodes_all / deals_total, "nodes_per_s": nodes_all / (elapsed_ms * 1e-3),
        "unsolved_results": unsolved,
        "helping_tasks": tasks,
        "warp_efficiency": eff,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": "ddg::batch_kernel",
                     "algorithmic_bytes": "TT bytes read+written per launch, counted in-kernel "
                                          f"({tt_bytes / max(1, nodes):.1f} B/node)"},
        "clocks": clocks,
        "gpu_launches": len(stats),
    }
    if e2e_ms:
        line["e2e"] = {"value": deals_total / (e2e_ms * 1e-3), "unit": "deals/s",
                       "h2d_bytes_per_step": B * 32, "d2h_bytes_per_step": B * 20}
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    solver.close()


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        reference_arm(a, rank, world)
        return
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


if __name__ == "__main__":
    main()
