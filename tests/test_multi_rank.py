"""Multi-GPU plumbing of bench.py on CPU: two `gloo` ranks take disjoint deal sets of the
same size (weak scaling, no data exchange) and combine their figures as the bench does
(max of the times, sum of the work)."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys
    sys.path.insert(0, ROOT)
    import datetime
    import torch
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        deals = bench.deal_set(rank)
        # per-rank figures: rank r took (r + 1) seconds and finished 100 (r + 1) jobs
        out = bench.combine_ranks(world, torch.device("cpu"), 1000.0 * (rank + 1), 500.0 * (rank + 1),
                                  100 * (rank + 1), 10 * (rank + 1), 1000 * (rank + 1))
        q.put((rank, deals[:64].tobytes(), deals.shape, out))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_combine():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        r, head, shape, out = q.get(timeout=120)
        res[r] = (np.frombuffer(head, dtype=np.uint64).reshape(-1, 4), shape, out)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (h0, s0, o0), (h1, s1, o1) = res[0], res[1]
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert s0 == s1 == (bench.SET_SIZE, 4)      # same work per rank (weak scaling)
    assert not (h0 == h1).all(axis=1).any()     # different deals
    assert o0 == o1                             # every rank gets the same combined figures
    elapsed, e2e, jobs, e2e_jobs, nodes = o0
    assert elapsed == 2000.0 and e2e == 1000.0  # the slowest rank's time
    assert jobs == 300 and e2e_jobs == 30 and nodes == 3000  # all ranks' work
