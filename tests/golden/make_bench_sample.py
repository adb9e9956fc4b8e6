"""Regenerates tests/golden/k13_bench_2000.npz: the reference solver's trick tables and
search-node counts for the first 2,000 deals of the 13-card benchmark set (seed 2, 13 cards
per seat, TT 2^10 buckets, one job per (deal, strain); dd_solve_strain, src/dd.h:926), run
by oracle/_ref/libddref.so (built by oracle/build_ref.sh from the reference's headers).

    python tests/golden/make_bench_sample.py [N]          # reference tables and nodes (CPU)
    python tests/golden/make_bench_sample.py guide [N]    # the guide's seeds and leads (GPU)
    python tests/golden/make_bench_sample.py guided [N]   # the guided search's nodes (CPU)

The first and the last take about 15 and 25 minutes on 8 cores. The fixture pins the
benchmark's results at scale (every job of these deals the GPU finishes is compared with
it) and gives the workload's search nodes per deal, which the benchmark uses to turn nodes
per second into deals per second.
"""
import ctypes
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
from deals_np import make_deals  # noqa: E402

P = ctypes.c_void_p


def guide_predictions(n):
    """The learned guide's NS seeds and root leads for the same deals, as the benchmark's
    guided run computes them on the GPU (needs a CUDA device and the weights file):
    tests/golden/k13_bench_N_guide.npz. With these the host replay of the solver's stage
    machine (tests/native/host_replay.cpp) gives the guided search's nodes per deal."""
    import torch
    sys.path.insert(0, ROOT)
    import dds_gpu_b200 as ddg
    from dds_gpu_b200 import guide
    params = guide.load_weights()
    assert params is not None, "no guide weights file"
    hands = make_deals(2, 0, n, 13)
    d_h = torch.from_numpy(hands.view(np.int64)).cuda()
    d_seed = torch.empty(n * 20, dtype=torch.int8, device="cuda")
    d_hint = torch.empty(n * 20, dtype=torch.int8, device="cuda")
    g = ddg.Guide(device=0, max_rows=8192, params=params)
    try:
        g.predict(d_h.data_ptr(), n, d_seed.data_ptr(), d_hint.data_ptr())
    finally:
        g.close()
    name = f"k13_bench_{n}_guide.npz"
    np.savez_compressed(os.path.join(HERE, name), seeds=d_seed.cpu().numpy().reshape(n, 5, 4),
                        hints=d_hint.cpu().numpy().reshape(n, 5, 4),
                        params_sum=np.float64(params.astype(np.float64).sum()))
    print(f"{name}: guide seeds and root leads for {n} deals")


def guided_nodes(n):
    """The guided search's node count per job for the same deals: the solver's own stage
    machine compiled for the host (tests/native/host_replay.cpp, node for node the GPU
    kernel's, as the tests check) stepping from the guide's seeds with its root leads first:
    tests/golden/k13_bench_N_guided.npz. Its tables must equal the reference's."""
    import subprocess
    src = os.path.join(ROOT, "tests", "native", "host_replay.cpp")
    lib_path = os.path.join(ROOT, "tests", "native", "_build", "libreplay_sample.so")
    os.makedirs(os.path.dirname(lib_path), exist_ok=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-fPIC", "-shared", "-Wno-unknown-pragmas",
                    "-I" + os.path.join(ROOT, "dds_gpu_b200", "csrc"), "-o", lib_path, src], check=True)
    lib = ctypes.CDLL(lib_path)
    with np.load(os.path.join(HERE, f"k13_bench_{n}_guide.npz")) as z:
        seeds = np.ascontiguousarray(z["seeds"], dtype=np.int8).reshape(-1)
        hints = np.ascontiguousarray(z["hints"], dtype=np.int8).reshape(-1)
        params_sum = float(z["params_sum"])
    with np.load(os.path.join(HERE, f"k13_bench_{n}.npz")) as z:
        want = z["tricks"]
    hands = make_deals(2, 0, n, 13)
    out = np.zeros(n * 20, np.int32)
    nodes = np.zeros(n * 5, np.uint64)
    t0 = time.time()
    rc = lib.replay_solve_hinted(hands.ctypes.data_as(P), ctypes.c_longlong(n), 10, 5, 1, seeds.ctypes.data_as(P),
                                 hints.ctypes.data_as(P), os.cpu_count() or 8, out.ctypes.data_as(P),
                                 nodes.ctypes.data_as(P), None)
    assert rc == 0
    tricks = out.reshape(n, 5, 4).astype(np.uint8)
    assert (tricks == want).all(), "the guided search changed a result"
    assert nodes.max() < 2**32
    name = f"k13_bench_{n}_guided.npz"
    np.savez_compressed(os.path.join(HERE, name), seed=2, k=13, tt_log2=10, tricks=tricks,
                        nodes_jpd5=nodes.astype(np.uint32), params_sum=np.float64(params_sum))
    print(f"{name}: {n} deals, {int(nodes.sum())} nodes ({nodes.sum() / n / 1e6:.2f} M per deal), "
          f"{time.time() - t0:.0f} s")


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "guide":
        guide_predictions(int(sys.argv[2]) if len(sys.argv) > 2 else 2000)
        return
    if len(sys.argv) > 1 and sys.argv[1] == "guided":
        guided_nodes(int(sys.argv[2]) if len(sys.argv) > 2 else 2000)
        return
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 2000
    ref = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libddref.so"))
    hands = make_deals(2, 0, n, 13)
    out = np.zeros(n * 20, np.int32)
    nodes = np.zeros(n * 5, np.uint64)
    t0 = time.time()
    rc = ref.ref_solve_batch(hands.ctypes.data_as(P), ctypes.c_long(n), 10, os.cpu_count() or 8,
                             out.ctypes.data_as(P), nodes.ctypes.data_as(P))
    assert rc == 0
    assert nodes.max() < 2**32
    name = f"k13_bench_{n}.npz"
    np.savez_compressed(os.path.join(HERE, name), seed=2, k=13, tt_log2=10, hands=hands,
                        tricks=out.reshape(n, 5, 4).astype(np.uint8), nodes_jpd5=nodes.astype(np.uint32))
    print(f"{name}: {n} deals, {int(nodes.sum())} nodes ({nodes.sum() / n / 1e6:.2f} M per deal), "
          f"{time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()
