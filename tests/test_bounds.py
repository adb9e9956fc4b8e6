"""The bounds-checked build (-DDDG_BOUNDS_CHECK): every frame-stack, TT-bucket and task
index of the stage machine is checked before its access, a failed check is counted and the
access skipped (no trap). On the CPU, the stage machine compiled with the checks searches
exactly as without them, and a stack deliberately too small for the endings (a planted
fault, on the host) is caught and counted. On the GPU, libddg_check.so solves the
fixtures with no check failing and the reference's tables."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import NATIVE, ROOT, load_golden

P = ctypes.c_void_p
CSRC = os.path.join(ROOT, "dds_gpu_b200", "csrc")


def build_replay(name, defines):
    src = os.path.join(NATIVE, "host_replay.cpp")
    out = os.path.join(NATIVE, "_build", name)
    os.makedirs(os.path.dirname(out), exist_ok=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-fPIC", "-shared", "-Wno-unknown-pragmas",
                    "-I" + CSRC] + defines + ["-o", out + ".tmp", src], check=True)
    os.replace(out + ".tmp", out)
    return ctypes.CDLL(out)


def replay(lib, hands, jpd=5):
    n = hands.shape[0]
    h = np.ascontiguousarray(hands, dtype=np.uint64)
    out = np.full(n * 20, -1, np.int32)
    nodes = np.zeros(n * jpd, np.uint64)
    stats = np.zeros(13, np.uint64)
    rc = lib.replay_solve(h.ctypes.data_as(P), ctypes.c_longlong(n), 10, jpd, 0, None, 8, out.ctypes.data_as(P),
                          nodes.ctypes.data_as(P), stats.ctypes.data_as(P))
    assert rc == 0
    return out.reshape(n, 5, 4), nodes, int(stats[12])


@pytest.fixture(scope="module")
def checked_replay():
    return build_replay("libreplay_check.so", ["-DDDG_BOUNDS_CHECK"])


def test_checks_change_nothing(checked_replay):
    for name, jpd in (("k9_120.npz", 5), ("k5_120.npz", 20)):
        g = load_golden(name)
        t, nodes, faults = replay(checked_replay, g["hands"], jpd)
        assert faults == 0
        assert (t == g["tricks"]).all() and (nodes == g[f"nodes_jpd{jpd}"]).all()


def test_planted_small_stack_is_caught():
    """A 12-frame stack holds the root and 11 plies. The last trick is decided at its lead
    without moves, so a K-card ending pushes 4 (K - 1) frames: 3-card endings (8) fit,
    5-card endings (16) do not; their lanes stop at the first push past the end."""
    lib = build_replay("libreplay_stack12.so", ["-DDDG_BOUNDS_CHECK", "-DDDG_STACK_DEPTH=12"])
    g = load_golden("k3_120.npz")
    t, _, faults = replay(lib, g["hands"])
    assert faults == 0 and (t == g["tricks"]).all()
    g = load_golden("k5_120.npz")
    t, _, faults = replay(lib, g["hands"][:20])
    assert faults > 0
    assert (t == -1).any()  # the stopped lanes left their results unwritten


@pytest.mark.gpu
def test_checked_library_on_the_gpu(ddg):
    import torch
    lib = ddg.load_library(ddg.CHECK_LIB_PATH)
    assert b"bounds-checked" in lib.ddg_version()
    for name, kw in (("k6_4096.npz", {}), ("k9_120.npz", {"jobs_per_deal": 20}),
                     ("k8_120.npz", {"schedule": 1, "block": 256, "min_blocks": 2}),
                     ("k7_120.npz", {"help": 1, "jobs_per_deal": 20, "lanes": 1024, "block": 256,
                                     "min_blocks": 2, "time_limit_s": 120})):
        g = load_golden(name)
        s = ddg.Solver(tt_log2=10, library=lib, **kw)
        try:
            n = g["hands"].shape[0]
            d_h = torch.from_numpy(g["hands"].view(np.int64)).cuda()
            d_o = torch.empty(n * 20, dtype=torch.uint8, device="cuda")
            st = s.solve_device(d_h.data_ptr(), n, d_o.data_ptr())  # raises if a check failed
            assert (d_o.cpu().numpy().reshape(n, 5, 4) == g["tricks"]).all(), name
            assert st["jobs_done"] == n * s.jobs_per_deal
        finally:
            s.close()
    m = load_golden("mixed_300.npz")
    mx = m["nodes_jpd5"].astype(np.int64).reshape(-1, 5).max(axis=1)
    sel = np.where(mx < 3_000_000)[0]
    hands = np.ascontiguousarray(m["hands"][sel])
    s = ddg.Solver(tt_log2=10, library=lib)
    try:
        assert (s.solve(hands) == m["tricks"][sel]).all()
    finally:
        s.close()
