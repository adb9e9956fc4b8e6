"""Serving load generator for the streaming solver (continuous batching, ddg_stream_*).

    python -m dds_gpu_b200.serve [--seconds 120] [--fractions 0.25,0.5,0.75,1.0]
                                 [--modes plain,guided] [--out FILE] [--sample-every 50]

Workload: a seeded mix of 70 % random 13-card deals and 30 % K-card endings, K uniform in
7..10, arriving as a Poisson process at fractions of the measured capacity. Capacity is
the stream's deal rate at full load: the node rate of every lane busy on the mix (a
saturated resumable solve) over the mix's mean nodes per deal (0.7 x 13.86 M for the
13-card deals, from complete reference solves of 2,000 of them, + 0.3 x 35 k for the
endings; --nodes-per-deal). The stream keeps a device ring of 65,536 deal slots and
admits deals as slots and lanes free up; deals that arrive while others are on the GPU
start as soon as a lane is free (continuous batching).

For each rate: deals arrive for --seconds (after --prefill deals at t = 0, if given);
solved rate, in-flight deals (sampled every
second) and the latency of every deal from its arrival to its result on the host, with
p50 / p99 / p99.9 over the deals that arrived in the second half of the window (after the
start-up) and finished before the drain limit; deals still running then are counted, not
guessed. Every --sample-every-th deal's table is kept (deal, table) for checking. Each
rate runs plain (DDS order, binary search) and guided (the learned guide's seeds and root
leads, computed on the GPU as deals are submitted), on the same lanes.
"""
import argparse
import json
import time

import numpy as np

from . import Solver, Stream, make_deals

MIX_SEED = 2026
NODES_PER_DEAL = 0.7 * 13.86e6 + 0.3 * 35e3


def mix_deals(seed, n):
    """n deals of the mix, in arrival order: (hands (n, 4) uint64, K per deal)."""
    rng = np.random.default_rng(seed)
    full = rng.random(n) < 0.7
    ks = np.where(full, 13, rng.integers(7, 11, n))
    hands = np.zeros((n, 4), dtype=np.uint64)
    for k in np.unique(ks):
        idx = np.where(ks == k)[0]
        hands[idx] = make_deals(seed + int(k), 0, len(idx), int(k))
    return hands, ks


def capacity(solver, seconds, torch):
    """Node rate with every lane busy on the mix (one resumable solve, a warm-up slice then
    a measured one) and the deal rate it gives."""
    hands, _ = mix_deals(MIX_SEED + 1, max(4 * solver.lanes // 5, 1000))
    n = hands.shape[0]
    d_h = torch.from_numpy(hands.view(np.int64)).cuda()
    d_o = torch.empty(n * 20, dtype=torch.uint8, device="cuda")
    solver.begin(d_h.data_ptr(), n, d_o.data_ptr())
    solver.resume(1.0)
    _, st = solver.resume(seconds)
    return st["nodes"] / (st["kernel_ms"] * 1e-3)


def arrival_times(rate, seconds, seed, prefill=0):
    """Arrival times (s, sorted): `prefill` deals at t = 0 (a backlog that brings the
    stream near its steady in-flight count sooner), then a Poisson process of `rate`
    deals/s up to `seconds`."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, int(rate * seconds * 1.5) + 100)
    arrivals = np.cumsum(gaps)
    return np.concatenate([np.zeros(prefill), arrivals[arrivals < seconds]])


def run_rate(solver, rate, seconds, drain_s, sample_every, seed, guide=None, prefill=0):
    arrivals = arrival_times(rate, seconds, seed, prefill)
    n = len(arrivals)
    hands, ks = mix_deals(seed, n)
    done_at = np.full(n, np.nan)
    sample = {}
    st = Stream(solver, ring_slots=65536, idle_timeout_s=5, guide=guide)
    in_flight = []
    submitted = 0
    t0 = time.perf_counter()
    next_tick = 1.0
    try:
        while True:
            now = time.perf_counter() - t0
            due = int(np.searchsorted(arrivals, now, side="right"))
            if submitted < due:
                submitted += st.submit(hands[submitted:due])
            idx, tab = st.poll()
            if len(idx):
                t = time.perf_counter() - t0
                for i, row in zip(idx.tolist(), tab):
                    done_at[i] = t
                    if i % sample_every == 0:
                        sample[i] = row.copy()
            if now >= next_tick:
                in_flight.append((round(now, 1), int(st.in_flight)))
                next_tick += 1.0
            if now >= seconds and (submitted >= n and (np.isfinite(done_at).all() or now >= seconds + drain_s)):
                break
            if not len(idx):
                time.sleep(0.0005)
    finally:
        stats = st.close(drain=False)
    lat = done_at - arrivals
    second_half = arrivals >= seconds / 2  # never a prefilled deal (they arrive at 0)
    fin = second_half & np.isfinite(lat)
    q = (lambda p: float(np.quantile(lat[fin], p) * 1e3)) if fin.any() else (lambda p: None)
    in_window = np.isfinite(done_at) & (done_at <= seconds)
    half = np.isfinite(done_at) & (done_at > seconds / 2) & (done_at <= seconds)
    mid = [v for t, v in in_flight if t <= seconds / 2]
    end = [v for t, v in in_flight if t <= seconds]
    return {
        "arrival_rate": rate, "prefill": int(prefill), "arrived": int(n), "admitted": int(submitted),
        "solved_in_window": int(in_window.sum()), "solved_rate_2nd_half": float(half.sum() / (seconds / 2)),
        "arrived_rate_2nd_half": float(second_half.sum() / (seconds / 2)),
        "in_flight_mid": mid[-1] if mid else None, "in_flight_end": end[-1] if end else None,
        "latency_ms": {"p50": q(0.5), "p99": q(0.99), "p999": q(0.999),
                       "deals": int(fin.sum()), "unfinished": int((second_half & ~np.isfinite(lat)).sum())},
        "latency_ms_endings": (float(np.median(lat[fin & (ks < 13)]) * 1e3) if (fin & (ks < 13)).any() else None),
        "latency_ms_full": (float(np.median(lat[fin & (ks == 13)]) * 1e3) if (fin & (ks == 13)).any() else None),
        "nodes": int(stats["nodes"]) if stats else None, "kernel_launches": int(stats["tasks"]) if stats else None,
        "sample": {int(i): row.reshape(-1).tolist() for i, row in sample.items()},
        "seed": seed,
    }


def main(argv=None):
    import torch
    p = argparse.ArgumentParser()
    p.add_argument("--seconds", type=float, default=120.0)
    p.add_argument("--drain", type=float, default=60.0, help="seconds to wait for late deals after the window")
    p.add_argument("--fractions", default="0.25,0.5,0.75,1.0")
    p.add_argument("--nodes-per-deal", type=float, default=NODES_PER_DEAL)
    p.add_argument("--capacity", type=float, default=0.0, help="deals/s at full load (0 = measure it)")
    p.add_argument("--sample-every", type=int, default=50)
    p.add_argument("--modes", default="plain,guided", help="plain and/or guided (the learned guide in the stream)")
    p.add_argument("--free-below", type=int, default=0, help="the solver's free_below (0 = its default)")
    p.add_argument("--prefill", type=int, default=0,
                   help="deals of the mix submitted at t = 0 before the Poisson arrivals (a backlog that "
                        "brings the stream near its steady state sooner; not in the latency figures)")
    p.add_argument("--out", default="")
    a = p.parse_args(argv)
    from . import Guide
    from .guide import load_weights
    # Both modes run on the same lanes: a guided stream leaves two SMs to the guide's kernels.
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    solver = Solver(tt_log2=10, jobs_per_deal=5, lanes=(sms - 2) * 512, free_below=a.free_below)
    guide = None
    try:
        cap = a.capacity
        rep = {"workload": "70% random 13-card deals + 30% K=7..10 endings, seeded, Poisson arrivals",
               "lanes": solver.lanes}
        if cap <= 0:
            nps = capacity(solver, 4.0, torch)
            cap = nps / a.nodes_per_deal
            rep["capacity_nodes_per_s"] = nps
        rep["capacity_deals_per_s"] = cap
        rep["rates"] = []
        modes = a.modes.split(",")
        params = load_weights() if "guided" in modes else None
        if params is not None:
            guide = Guide(device=0, max_rows=4096, params=params)
        for i, f in enumerate(float(x) for x in a.fractions.split(",")):
            for mode in modes:
                if mode == "guided" and guide is None:
                    continue
                r = run_rate(solver, f * cap, a.seconds, a.drain, a.sample_every, MIX_SEED + 100 + i,
                             guide if mode == "guided" else None, a.prefill)
                r["fraction"] = f
                r["mode"] = mode
                rep["rates"].append(r)
                print(json.dumps({k: v for k, v in r.items() if k != "sample"}), flush=True)
    finally:
        if guide is not None:
            guide.close()
        solver.close()
    if a.out:
        with open(a.out, "w") as f:
            json.dump(rep, f)
    return rep


if __name__ == "__main__":
    main()
