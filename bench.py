#!/usr/bin/env python
"""Benchmark: exact double-dummy deals/s on B200s (one process per GPU, weak scaling).

Workload: the 13-card benchmark set, 20,000 seeded uniformly random deals per GPU
(ddg_make_deals seed 2; rank r takes deals [20000 r, 20000 (r+1)) of that stream), one
job per (deal, strain) with the four declarers sharing a TT of 2^10 buckets, all inputs
resident in HBM. The set is solved as one resumable solve (ddg_solve_begin); one step is
one slice of it (ddg_solve_continue, --slice-s seconds, every lane's search state kept in
HBM between slices), so each step is one kernel launch timed with CUDA events.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Rank 0 prints one JSON line. `value` = (deal, strain) jobs finished by all ranks in the K
timed slices / 5 / max over ranks of the timed device time: the reference's own headline
metric ("full-job deals/s": finished jobs / 5 per second while the set is being solved),
with the learned guide's seeds and root leads when its weights file is there (`plain` =
the same measurement without the guide, run first on the same set).
Only finished, exact jobs count; work in progress at the end of the timed slices does
not. `e2e` = the same through the host API with, every step, the deals copied in from
pinned host memory and all results copied out. `roofline` = TT bytes the search moved
(counted in-kernel) per second of kernel time, against the measured HBM copy bandwidth.
`cpu_baseline` = the reference's own CPU solver (compiled from its sources into
oracle/_ref, else the C restatement) on the same deals over the same slices, all host
cores. `--impl reference` prints that CPU measurement as the reference arm.
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
SET_SEED, SET_SIZE, SET_K = 2, 20000, 13
JPD = 5
DRAM_BYTES_PER_NODE = 53.9  # dram__bytes_read.sum + dram__bytes_write.sum per node, 13-card slice
WORKLOAD = ("13-card seeded random deals (20,000 per GPU), all 5 strains x 4 declarers, "
            "exact TT 2^10 buckets per lane, one job per (deal, strain)")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--slice-s", type=float, default=4.0, help="seconds per step (one slice of the solve)")
    p.add_argument("--tt-log2", type=int, default=10)
    p.add_argument("--lanes", type=int, default=0, help="0 = fill the GPU")
    p.add_argument("--block", type=int, default=0, help="threads (lanes) per block; 0 = library default (512)")
    p.add_argument("--min-blocks", type=int, default=0)
    p.add_argument("--schedule", type=int, default=0, help="0 block-phase kernel, 1 queue kernel")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-guide", action="store_true", help="plain solver only (no learned guide)")
    return p.parse_args()


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def deal_set(rank):
    from dds_gpu_b200 import make_deals
    return make_deals(SET_SEED, rank * SET_SIZE, SET_SIZE, SET_K)


# ---- CPU reference path (baseline only) -------------------------------------------------

def cpu_window(deals, tt_log2, slice_s, slices):
    """The reference's CPU solver over the deal set for `slices` slices of `slice_s` seconds
    (oracle/_ref/cpu_window, built from the reference's sources; else the C restatement's
    oracle/_build/cpu_window). Returns (jobs finished per slice, nodes per slice, threads, kind)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "cpu_window")
    if not os.path.exists(exe):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
        exe = os.path.join(ROOT, "oracle", "_build", "cpu_window")
    cores = host_cores()
    with tempfile.NamedTemporaryFile(suffix=".bin", delete=False) as f:
        f.write(deals.tobytes())
        path = f.name
    try:
        out = subprocess.run([exe, path, str(tt_log2), str(cores), str(slice_s), str(slices)],
                             check=True, capture_output=True, text=True,
                             timeout=slice_s * slices + 120).stdout
    finally:
        os.unlink(path)
    r = json.loads(out.strip().splitlines()[-1])
    return r["jobs"], r["nodes"], r["threads"], r["kind"]


def cpu_measure(a, deals):
    jobs, nodes, threads, kind = cpu_window(deals, a.tt_log2, a.slice_s, a.warmup + a.steps)
    t_jobs = sum(jobs[a.warmup:])
    value = t_jobs / JPD / (a.steps * a.slice_s)
    sample = (f"deal set seed {SET_SEED} (20,000 deals) solved by {threads} threads, one TT each; "
              f"(deal, strain) jobs finished in slices {a.warmup}..{a.warmup + a.steps - 1} of "
              f"{a.slice_s:g} s (first {a.warmup} = warm-up): {t_jobs} jobs, "
              f"{sum(nodes[a.warmup:]) / max(1, t_jobs):.0f} nodes/job")
    return {"value": value, "unit": "deals/s", "cores": threads, "kind": kind, "sample": sample}


def config_dict(a, world, extra=None):
    d = {"workload": WORKLOAD, "deal_set": f"seed {SET_SEED}, {SET_SIZE} deals per GPU, K={SET_K}",
         "tt_log2": a.tt_log2, "jobs_per_deal": JPD, "step": f"one {a.slice_s:g} s slice of the resumable solve",
         "parallelism": f"dp{world} (own deal set per GPU, no collective on the data path)",
         "l2": "flushed between steps (256 MiB write); the TT working set (GBs) is far above L2"}
    if extra:
        d.update(extra)
    return d


def reference_arm(a, rank, world):
    if rank != 0:
        return
    cpu = cpu_measure(a, deal_set(0))
    line = {"metric": METRIC, "value": cpu["value"], "unit": "deals/s", "impl": "reference", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * a.slice_s,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic", "config": config_dict(a, world),
            "cpu_baseline": cpu,
            "e2e": {"value": cpu["value"], "unit": "deals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
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


def golden_check(tables):
    """Results the GPU finished for the first deals of the set (rank 0's) against the
    reference's tables in the committed fixture (tests/golden/k13_24.npz)."""
    import numpy as np
    g = np.load(os.path.join(ROOT, "tests", "golden", "k13_24.npz"))
    want = g["tricks"].reshape(-1, 20)
    got = tables[: want.shape[0]]
    done = got != 255
    return {"checked": int(done.sum()), "equal": bool((got[done] == want[done]).all())}


def our_arm(a, rank, world, local_rank):
    import numpy as np
    import torch
    import dds_gpu_b200 as ddg
    import dds_gpu_b200.guide as ddg_guide

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    deals = deal_set(rank)
    solver = ddg.Solver(tt_log2=a.tt_log2, lanes=a.lanes, block=a.block, jobs_per_deal=JPD, device=local_rank,
                        min_blocks=a.min_blocks, schedule=a.schedule)
    n = deals.shape[0]
    host_in = torch.from_numpy(deals.view(np.int64)).pin_memory()
    dev_in = host_in.to(dev)
    dev_out = torch.empty((n, 20), dtype=torch.uint8, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    cs = stream.cuda_stream

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def window(d_seed=0, d_hint=0):
        """W warm-up and K timed slices of one resumable solve of the set."""
        solver.begin(dev_in.data_ptr(), n, dev_out.data_ptr(), d_seeds=d_seed, d_hints=d_hint, stream=cs)
        for s in range(a.warmup):  # warm-up slices (untimed)
            flush.zero_()
            solver.resume(a.slice_s, stream=cs)
        torch.cuda.synchronize(dev)
        sampler = ClockSampler(local_rank)
        stats = []
        barrier()
        torch.cuda.synchronize(dev)
        sampler.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for s in range(a.steps):
            flush.zero_()
            stats.append(solver.resume(a.slice_s, stream=cs)[1])
        e1.record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        return stats, e0.elapsed_time(e1), sampler.stop(), dev_out.cpu().numpy()

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
        guide_ms = 1e3 * (time.perf_counter() - g0)
        guide.close()
        guide_info = {"predict_ms": guide_ms, "rows": n * 20}

    plain_stats, plain_ms, plain_clocks, plain_tables = window()
    plain_jobs = sum(st["jobs_done"] for st in plain_stats)
    if d_seed is not None:
        stats, elapsed_ms, clocks, tables = window(d_seed.data_ptr(), d_hint.data_ptr())
        seeds = d_seed.cpu().numpy().reshape(n, 5, 4).astype(int)
        t = tables.reshape(n, 5, 4).astype(int)
        ns = np.where(np.arange(4) % 2 == 0, t, 13 - t)
        done = t <= 13
        guide_info.update({"seed_exact": float((seeds == ns)[done].mean()) if done.any() else None,
                           "seed_within_one": float((abs(seeds - ns) <= 1)[done].mean()) if done.any() else None})
    else:
        stats, elapsed_ms, clocks, tables = plain_stats, plain_ms, plain_clocks, plain_tables
    jobs = sum(st["jobs_done"] for st in stats)
    # equal tables where both runs finished: the guide changes the work, never an answer
    both = (plain_tables != 255) & (tables != 255)
    guided_equal_plain = bool((plain_tables[both] == tables[both]).all())

    # End to end through the host API: each step copies the deals in from pinned host memory,
    # runs the slice and copies every result out.
    e2e_ms, e2e_jobs = None, 0
    if not a.no_e2e:
        host_out = torch.empty((n, 20), dtype=torch.uint8).pin_memory()
        solver.begin(dev_in.data_ptr(), n, dev_out.data_ptr(), stream=cs,
                     d_seeds=d_seed.data_ptr() if d_seed is not None else 0,
                     d_hints=d_hint.data_ptr() if d_hint is not None else 0)
        for s in range(a.warmup):
            solver.resume(a.slice_s, hands_host=host_in.data_ptr(), out_host=host_out.data_ptr(), stream=cs)
        barrier()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for s in range(a.steps):
            flush.zero_()
            e2e_jobs += solver.resume(a.slice_s, hands_host=host_in.data_ptr(), out_host=host_out.data_ptr(),
                                      stream=cs)[1]["jobs_done"]
            assert int((host_out[:24] != 255).sum()) >= 0  # the results are on the host
        torch.cuda.synchronize(dev)
        e2e_ms = 1e3 * (time.perf_counter() - t0)
        barrier()

    nodes = sum(st["nodes"] for st in stats)
    elapsed_ms, e2e_ms, jobs_all, e2e_jobs_all, nodes_all = combine_ranks(
        world, dev, elapsed_ms, e2e_ms, jobs, e2e_jobs, nodes)
    plain_ms_all, _, plain_jobs_all, _, plain_nodes_all = combine_ranks(
        world, dev, plain_ms, None, plain_jobs, 0, sum(st["nodes"] for st in plain_stats))

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cpu = cpu_measure(a, deals)

    if rank != 0:
        solver.close()
        return
    kernel_ms = sum(st["kernel_ms"] for st in stats)
    tt_bytes = sum(st["tt_bytes"] for st in stats)
    it = [sum(st["phase_warps"][k] for st in stats) for k in range(5)]
    ln = [sum(st["phase_items"][k] for st in stats) for k in range(5)]
    peak, peak_kind = peaks()
    achieved = tt_bytes / (kernel_ms * 1e-3) / 1e9 if kernel_ms else 0.0
    value = jobs_all / JPD / (elapsed_ms * 1e-3)
    eff = {name: (ln[k] / (32.0 * it[k]) if it[k] else None)
           for k, name in enumerate(["cheap", "enter_lead", "enter_follow", "moves_lead", "moves_follow"])}
    # DRAM bytes per launch: the per-node DRAM traffic of one ncu capture of this kernel on a
    # smaller case of the same workload (profiles/batch_kernel_13card_full.md), scaled by
    # the nodes a bench launch searches.
    traffic = DRAM_BYTES_PER_NODE * nodes / max(1, len(stats))
    line = {
        "metric": METRIC, "value": value, "unit": "deals/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": elapsed_ms / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
        "config": config_dict(a, world, {"lanes": stats[0]["lanes"] if stats else 0,
                                         "block": stats[0]["block"] if stats else a.block,
                                         "schedule": a.schedule,
                                         "guide": ("learned guide: NS seeds (stepping search) + root leads"
                                                   if guide_info else "off (plain DDS move order)")}),
        "jobs_finished": int(jobs_all), "nodes_per_s": nodes_all / (elapsed_ms * 1e-3),
        "nodes_per_finished_job": nodes_all / max(1, jobs_all),
        "plain": {"value": plain_jobs_all / JPD / (plain_ms_all * 1e-3), "unit": "deals/s",
                  "jobs_finished": int(plain_jobs_all),
                  "nodes_per_finished_job": plain_nodes_all / max(1, plain_jobs_all)},
        "guide": guide_info,
        "guided_tables_equal_plain": guided_equal_plain,
        "golden_check": golden_check(tables),
        "warp_efficiency": eff,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": f"ddg::batch_kernel<{solver.block_shape}>",
                     "algorithmic_bytes": "TT bytes read+written per launch, counted in-kernel "
                                          f"({tt_bytes / max(1, nodes):.1f} B/node)"},
        "clocks": clocks,
        "gpu_launches": len(stats),
    }
    if e2e_ms:
        line["e2e"] = {"value": e2e_jobs_all / JPD / (e2e_ms * 1e-3), "unit": "deals/s",
                       "h2d_bytes_per_step": n * 32, "d2h_bytes_per_step": n * 20}
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
