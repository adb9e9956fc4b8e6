"""GPU parity: the CUDA kernel against the reference's golden tables and node counts,
called through the C ABI (libddg.so). Bit-exact tricks; node counts equal one for one
because the search, bounds, move order and TT decisions are the reference's."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def device_solve(ddg, solver, hands, seeds=None):
    import torch
    n = hands.shape[0]
    d_h = torch.from_numpy(hands.view(np.int64)).cuda()
    d_o = torch.empty(n * 20, dtype=torch.uint8, device="cuda")
    d_nodes = torch.zeros(n * solver.jobs_per_deal, dtype=torch.int64, device="cuda")
    d_s = None
    if seeds is not None:
        d_s = torch.from_numpy(np.ascontiguousarray(seeds, dtype=np.int8).reshape(-1)).cuda()
    st = solver.solve_device(d_h.data_ptr(), n, d_o.data_ptr(), d_s.data_ptr() if d_s is not None else 0,
                             d_nodes.data_ptr())
    return d_o.cpu().numpy().reshape(n, 5, 4), d_nodes.cpu().numpy().view(np.uint64), st


@pytest.mark.parametrize("name", [f"k{k}_120.npz" for k in range(1, 10)] + ["k6_4096.npz"])
def test_endings_jpd5(ddg, gpu_solver, name):
    g = load_golden(name)
    t, nodes, st = device_solve(ddg, gpu_solver, g["hands"])
    assert (t == g["tricks"]).all()
    assert (nodes == g["nodes_jpd5"]).all()
    assert st["nodes"] == int(g["nodes_jpd5"].sum())
    assert st["jobs_done"] == g["hands"].shape[0] * 5


@pytest.fixture(scope="module")
def solver20(ddg):
    s = ddg.Solver(tt_log2=10, jobs_per_deal=20, lanes=16384)
    yield s
    s.close()


@pytest.mark.parametrize("name", ["k3_120.npz", "k6_4096.npz", "k9_120.npz"])
def test_endings_jpd20(ddg, solver20, name):
    g = load_golden(name)
    t, nodes, st = device_solve(ddg, solver20, g["hands"])
    assert (t == g["tricks"]).all()
    assert (nodes == g["nodes_jpd20"]).all()


LIGHT_13 = [1, 3, 15, 17, 22]  # full deals of the fixture whose largest job is < 600k nodes


def test_full_deals(ddg, gpu_solver):
    g = load_golden("k13_24.npz")
    hands = np.ascontiguousarray(g["hands"][LIGHT_13])
    t, nodes, st = device_solve(ddg, gpu_solver, hands)
    assert (t == g["tricks"][LIGHT_13]).all()
    want = g["nodes_jpd5"].reshape(-1, 5)[LIGHT_13].reshape(-1)
    assert (nodes == want).all()


@pytest.mark.parametrize("tt", [9, 12])
def test_tt_sizes(ddg, tt):
    g = load_golden(f"k7_200_tt{tt}.npz")
    s = ddg.Solver(tt_log2=tt, lanes=4096)
    try:
        t, nodes, _ = device_solve(ddg, s, g["hands"])
    finally:
        s.close()
    assert (t == g["tricks"]).all() and (nodes == g["nodes_jpd5"]).all()


def test_seeded_stepping(ddg, gpu_solver):
    g = load_golden("k8_200_seeded.npz")
    t, nodes, _ = device_solve(ddg, gpu_solver, g["hands"], g["seeds"])
    assert (t == g["tricks"]).all() and (nodes == g["nodes_jpd5"]).all()


def test_host_api_and_repeat_calls(ddg, gpu_solver):
    """Host-buffer call, called twice: same tables (TT generations carry over calls)."""
    g = load_golden("k7_120.npz")
    a = gpu_solver.solve(g["hands"])
    b = gpu_solver.solve(g["hands"])
    assert (a == g["tricks"]).all() and (b == g["tricks"]).all()
    assert gpu_solver.last_stats["nodes"] == int(g["nodes_jpd5"].sum())


def test_generation_wrap(ddg):
    """More than 63 jobs per lane: the TT generation wraps and the tags are cleared."""
    g = load_golden("k5_120.npz")
    s = ddg.Solver(tt_log2=9, lanes=64, block=64)
    try:
        for _ in range(3):
            t, nodes, _ = device_solve(ddg, s, g["hands"])
            assert (t == g["tricks"]).all() and (nodes == g["nodes_jpd5"]).all()
    finally:
        s.close()


def test_solve_strain_matches_batch(ddg, gpu_solver):
    g = load_golden("k6_120.npz")
    for i in range(4):
        for strain in range(5):
            out4 = gpu_solver.solve_strain(g["hands"][i], strain)
            assert out4 == [int(x) for x in g["tricks"][i, strain]]


def test_empty_batch_and_bad_input(ddg, gpu_solver):
    out = gpu_solver.solve(np.zeros((0, 4), np.uint64))
    assert out.shape == (0, 5, 4)
    bad = load_golden("k4_120.npz")["hands"][:3].copy()
    bad[1, 0] = bad[1, 1]
    with pytest.raises(ddg.DDGError):
        gpu_solver.solve(bad)
    with pytest.raises(ddg.DDGError):
        gpu_solver.solve_strain(load_golden("k4_120.npz")["hands"][0], 5)


def test_ragged_batch_sizes(ddg, gpu_solver):
    """Batches that are not multiples of a block or warp, down to one deal."""
    g = load_golden("k8_120.npz")
    for n in (1, 31, 33, 97):
        t = gpu_solver.solve(g["hands"][:n])
        assert (t == g["tricks"][:n]).all()


@pytest.fixture(scope="module")
def helper_solver(ddg):
    # helpers in their own TTs (help_share_tt = -1); the shared-TT default is tested below
    s = ddg.Solver(tt_log2=10, jobs_per_deal=20, lanes=1024, block=256, min_blocks=2, help=1, help_share_tt=-1,
                   time_limit_s=120)
    yield s
    s.close()


@pytest.mark.parametrize("name", ["k5_120.npz", "k7_120.npz", "k9_120.npz", "k6_4096.npz"])
def test_helping_exact_tricks(ddg, helper_solver, name):
    """With helping on, idle lanes take over sibling moves of busy lanes: node counts change,
    every trick count must still equal the reference's."""
    g = load_golden(name)
    t, _, st = device_solve(ddg, helper_solver, g["hands"])
    assert (t == g["tricks"]).all()
    assert st["jobs_done"] == g["hands"].shape[0] * 20


@pytest.mark.parametrize("name", ["k7_120.npz", "k9_120.npz", "k6_4096.npz"])
def test_shared_tt_helping_exact_tricks(ddg, name):
    """Helpers search their tasks in the donor's TT, which the donor and every helper of the
    job read and write at once (sealed entries make a torn entry a miss): tricks exact."""
    g = load_golden(name)
    s = ddg.Solver(tt_log2=10, jobs_per_deal=20, lanes=1024, block=256, min_blocks=2, help=1, help_share_tt=1,
                   time_limit_s=120)
    try:
        t, _, st = device_solve(ddg, s, g["hands"])
        assert (t == g["tricks"]).all()
        assert st["jobs_done"] == g["hands"].shape[0] * 20
        hard = load_golden("k13_24.npz")
        t, _, st = device_solve(ddg, s, np.ascontiguousarray(hard["hands"][LIGHT_13]))
        assert (t == hard["tricks"][LIGHT_13]).all() and st["tasks"] > 0
    finally:
        s.close()


def test_helping_splits_hard_deals(ddg, helper_solver):
    """Few full deals on many lanes: lanes go hungry at once and take donated moves."""
    g = load_golden("k13_24.npz")
    hands = np.ascontiguousarray(g["hands"][LIGHT_13])
    t, _, st = device_solve(ddg, helper_solver, hands)
    assert (t == g["tricks"][LIGHT_13]).all()
    assert st["tasks"] > 0


@pytest.mark.parametrize("schedule", [0, 1])
def test_resumable_slices(ddg, schedule):
    """A solve cut into short slices (lane states kept in HBM between launches) gives the
    reference's tricks and exactly the node counts of one uninterrupted solve."""
    import torch
    g = load_golden("k8_120.npz")
    n = g["hands"].shape[0]
    s = ddg.Solver(tt_log2=10, jobs_per_deal=5, lanes=2048, block=256, min_blocks=2, schedule=schedule)
    try:
        d_h = torch.from_numpy(g["hands"].view(np.int64)).cuda()
        d_o = torch.empty(n * 20, dtype=torch.uint8, device="cuda")
        s.begin(d_h.data_ptr(), n, d_o.data_ptr())
        nodes = jobs = slices = 0
        finished = False
        while not finished:
            finished, st = s.resume(0.002)
            nodes += st["nodes"]
            jobs += st["jobs_done"]
            slices += 1
            assert slices < 100000
        assert slices > 2
        assert (d_o.cpu().numpy().reshape(n, 5, 4) == g["tricks"]).all()
        assert nodes == int(g["nodes_jpd5"].astype(np.int64).sum())
        assert jobs == n * 5
        # a finished solve stays finished; a plain solve afterwards works as before
        assert s.resume(0.002)[0]
        t, _, _ = device_solve(ddg, s, g["hands"])
        assert (t == g["tricks"]).all()
    finally:
        s.close()


def test_queue_kernel_parity(ddg):
    """The barrier-free queue kernel (schedule 1) runs the same stages: same tricks and
    node counts as the reference."""
    g = load_golden("k6_4096.npz")
    s = ddg.Solver(tt_log2=10, jobs_per_deal=5, block=256, min_blocks=2, schedule=1)
    try:
        t, nodes, st = device_solve(ddg, s, g["hands"])
        assert (t == g["tricks"]).all()
        assert (nodes == g["nodes_jpd5"]).all()
    finally:
        s.close()


def test_stream_continuous_batching(ddg):
    """Deals submitted while others are on the GPU come back with the same tables as when
    each is solved alone (and as the reference's), out of order, each exactly once."""
    import time
    g = load_golden("k7_120.npz")
    hands, want = g["hands"], g["tricks"]
    s = ddg.Solver(tt_log2=10, jobs_per_deal=5, lanes=4096, block=256, min_blocks=2)
    try:
        # alone: one deal at a time
        st = ddg.Stream(s, ring_slots=64, idle_timeout_s=5)
        alone = np.zeros_like(want)
        for i in range(8):
            assert st.submit(hands[i:i + 1]) == 1
            t0 = time.time()
            while True:
                idx, tab = st.poll()
                if len(idx):
                    assert list(idx) == [i]
                    alone[i] = tab[0]
                    break
                assert time.time() - t0 < 60
        st.close()
        # in the mix: everything at once through a small ring (admission holds the rest back)
        st = ddg.Stream(s, ring_slots=64, idle_timeout_s=5)
        got = np.full_like(want, 255)
        seen = np.zeros(len(hands), dtype=int)
        sent = 0
        t0 = time.time()
        while seen.sum() < len(hands):
            if sent < len(hands):
                sent += st.submit(hands[sent:])
            idx, tab = st.poll()
            for k, i in enumerate(idx):
                seen[i] += 1
                got[i] = tab[k]
            assert time.time() - t0 < 120
        stats = st.close()
        assert (seen == 1).all()
        assert (got == want).all()
        assert (alone[:8] == got[:8]).all()
        assert stats["jobs_done"] == len(hands) * 5
        # the solver works normally after the stream is closed
        assert (s.solve(hands[:4]) == want[:4]).all()
    finally:
        s.close()


@pytest.mark.parametrize("block,min_blocks,schedule,cheap_limit,spread",
                         [(512, 1, 0, 0, 0), (256, 2, 0, 0, 0), (512, 1, 2, 0, 0), (512, 1, 0, -1, 0),
                          (512, 1, 0, 1, 0), (256, 2, 0, 0, 1), (128, 4, 0, 0, 0)])
def test_launch_shapes_and_schedules(ddg, block, min_blocks, schedule, cheap_limit, spread):
    """Every launch shape and stage schedule the autotuner may pick searches exactly the
    reference's nodes, job for job."""
    g = load_golden("k8_120.npz")
    s = ddg.Solver(tt_log2=10, jobs_per_deal=5, lanes=4096, block=block, min_blocks=min_blocks,
                   schedule=schedule, cheap_limit=cheap_limit, phase_spread=spread)
    try:
        t, nodes, st = device_solve(ddg, s, g["hands"])
        assert (t == g["tricks"]).all()
        assert (nodes == g["nodes_jpd5"]).all()
    finally:
        s.close()


@pytest.mark.parametrize("block,min_blocks,flat", [(512, 1, 1), (256, 2, 1), (512, 1, -1)])
def test_flat_lead_moves(ddg, block, min_blocks, flat):
    """The lead-move phase with its (lane, candidate) pairs spread over the block (the
    default) orders the moves as the per-lane loop (flat_moves = -1) does: both give the
    reference's tricks and node counts, job for job."""
    s = ddg.Solver(tt_log2=10, jobs_per_deal=5, lanes=4096, block=block, min_blocks=min_blocks, flat_moves=flat)
    try:
        for name in ("k8_120.npz", "k6_4096.npz"):
            g = load_golden(name)
            t, nodes, _ = device_solve(ddg, s, g["hands"])
            assert (t == g["tricks"]).all() and (nodes == g["nodes_jpd5"]).all(), name
        g = load_golden("k13_24.npz")
        hands = np.ascontiguousarray(g["hands"][LIGHT_13])
        t, nodes, _ = device_solve(ddg, s, hands)
        assert (t == g["tricks"][LIGHT_13]).all()
        assert (nodes == g["nodes_jpd5"].reshape(-1, 5)[LIGHT_13].reshape(-1)).all()
    finally:
        s.close()


@pytest.mark.parametrize("free_pack", [1, 8, 32])
def test_free_rounds_packing(ddg, free_pack):
    """Blocks that run only free-running rounds (free_below above the block size), with
    their busy lanes one to a warp (free_pack 1), eight to a warp, or packed into as few
    warps as hold them (32): which warp steps a lane changes nothing in its search, so the
    tricks and node counts are the reference's, job for job."""
    s = ddg.Solver(tt_log2=10, jobs_per_deal=5, lanes=4096, free_below=1024, free_pack=free_pack)
    try:
        for name in ("k8_120.npz", "k6_4096.npz"):
            g = load_golden(name)
            t, nodes, _ = device_solve(ddg, s, g["hands"])
            assert (t == g["tricks"]).all() and (nodes == g["nodes_jpd5"]).all(), name
        g = load_golden("k13_24.npz")
        hands = np.ascontiguousarray(g["hands"][LIGHT_13])
        t, nodes, _ = device_solve(ddg, s, hands)
        assert (t == g["tricks"][LIGHT_13]).all()
        assert (nodes == g["nodes_jpd5"].reshape(-1, 5)[LIGHT_13].reshape(-1)).all()
        assert s.last_stats["free_rounds"] > 0 and s.last_stats["phase_warps"] == [0] * 5
    finally:
        s.close()
