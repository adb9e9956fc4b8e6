"""The product's stage machine, replayed on the host, against the reference's golden tables
and node counts (tests/golden, made by the reference itself). Node counts agree only if
every bound, TT decision and move-order choice agrees, so this pins the GPU code's logic."""
import ctypes

import numpy as np
import pytest

from conftest import load_golden

P = ctypes.c_void_p


def replay(lib, hands, tt_log2=10, jpd=5, seeds=None, threads=8):
    n = hands.shape[0]
    h = np.ascontiguousarray(hands, dtype=np.uint64)
    out = np.zeros(n * 20, np.int32)
    nodes = np.zeros(n * jpd, np.uint64)
    sd = None if seeds is None else np.ascontiguousarray(seeds, dtype=np.int8).reshape(-1)
    rc = lib.replay_solve(h.ctypes.data_as(P), ctypes.c_longlong(n), tt_log2, jpd, 0 if seeds is None else 1,
                          None if sd is None else sd.ctypes.data_as(P), threads, out.ctypes.data_as(P),
                          nodes.ctypes.data_as(P), None)
    assert rc == 0
    return out.reshape(n, 5, 4), nodes


@pytest.mark.parametrize("name", [f"k{k}_120.npz" for k in range(1, 10)] + ["k6_4096.npz"])
@pytest.mark.parametrize("jpd", [5, 20])
def test_endings(replay_lib, name, jpd):
    g = load_golden(name)
    t, nodes = replay(replay_lib, g["hands"], int(g["tt_log2"]), jpd)
    assert (t == g["tricks"]).all()
    assert (nodes == g[f"nodes_jpd{jpd}"]).all()


def test_full_deals(replay_lib):
    g = load_golden("k13_24.npz")
    t, nodes = replay(replay_lib, g["hands"][:12])
    assert (t == g["tricks"][:12]).all()
    assert (nodes == g["nodes_jpd5"][:12 * 5]).all()


@pytest.mark.parametrize("tt", [9, 12])
def test_tt_sizes(replay_lib, tt):
    g = load_golden(f"k7_200_tt{tt}.npz")
    t, nodes = replay(replay_lib, g["hands"], tt)
    assert (t == g["tricks"]).all() and (nodes == g["nodes_jpd5"]).all()


def test_seeded_stepping(replay_lib):
    g = load_golden("k8_200_seeded.npz")
    t, nodes = replay(replay_lib, g["hands"], 10, 5, g["seeds"])
    assert (t == g["tricks"]).all() and (nodes == g["nodes_jpd5"]).all()
