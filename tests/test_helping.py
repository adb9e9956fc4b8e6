"""Helping (idle lanes take over donated sibling moves of busy lanes), run on the host by a
simulated block that steps its lanes through the GPU kernel's phases. Node counts change
with helping; every trick count must still equal the reference's, every task must return
to the pool and every helping counter must end at zero (the simulator checks both)."""
import ctypes

import numpy as np
import pytest

from conftest import load_golden

P = ctypes.c_void_p


def block(lib, hands, lanes, eager, jpd=5, tt_log2=10, free_below=0, free_steps=64, cheap_limit=0):
    n = hands.shape[0]
    h = np.ascontiguousarray(hands, dtype=np.uint64)
    out = np.zeros(n * 20, np.int32)
    st = np.zeros(14, np.uint64)
    rc = lib.replay_block(h.ctypes.data_as(P), ctypes.c_longlong(n), tt_log2, jpd, lanes, eager, free_below,
                          free_steps, out.ctypes.data_as(P), st.ctypes.data_as(P), cheap_limit)
    return rc, out.reshape(n, 5, 4), st


@pytest.mark.parametrize("name", ["k4_120.npz", "k6_120.npz", "k8_120.npz", "k9_120.npz"])
@pytest.mark.parametrize("lanes,eager,jpd,free", [(3, 1, 5, 0), (16, 0, 20, 0), (16, 1, 20, 0), (64, 1, 5, 0),
                                                  (16, 1, 20, 8), (64, 0, 5, 40), (32, 1, 20, 1000)])
def test_helping_keeps_tricks(replay_lib, name, lanes, eager, jpd, free):
    g = load_golden(name)
    rc, t, st = block(replay_lib, g["hands"][:48], lanes, eager, jpd, free_below=free, free_steps=17)
    assert rc == 0
    assert (t == g["tricks"][:48]).all()
    if eager:
        assert st[12] > 0  # tasks were donated


def test_helping_full_deals(replay_lib):
    g = load_golden("k13_24.npz")
    idx = [1, 3, 15]
    rc, t, st = block(replay_lib, g["hands"][idx], 32, 1, 20)
    assert rc == 0 and (t == g["tricks"][idx]).all() and st[12] > 0


@pytest.mark.parametrize("name", ["k6_120.npz", "k9_120.npz"])
@pytest.mark.parametrize("cheap_limit", [1, 2, 3])
@pytest.mark.parametrize("lanes,eager,jpd", [(16, 1, 20), (64, 1, 5), (32, 0, 20)])
def test_helping_with_cheap_limit(replay_lib, name, cheap_limit, lanes, eager, jpd):
    """The GPU kernel's cheap pass stops a lane after a few stages; helping must stay exact
    when a lane is left mid-chain (in NEXT, RET, WAIT or HUNGRY) between passes."""
    g = load_golden(name)
    rc, t, st = block(replay_lib, g["hands"][:48], lanes, eager, jpd, cheap_limit=cheap_limit)
    assert rc == 0
    assert (t == g["tricks"][:48]).all()


def block_shared(lib, hands, lanes, eager, jpd=5, cheap_limit=0, free_below=0):
    n = hands.shape[0]
    h = np.ascontiguousarray(hands, dtype=np.uint64)
    out = np.zeros(n * 20, np.int32)
    st = np.zeros(14, np.uint64)
    rc = lib.replay_block_ex(h.ctypes.data_as(P), ctypes.c_longlong(n), 10, jpd, lanes, eager, free_below, 17,
                             out.ctypes.data_as(P), st.ctypes.data_as(P), cheap_limit, 1)
    return rc, out.reshape(n, 5, 4), st


@pytest.mark.parametrize("name", ["k5_120.npz", "k8_120.npz", "k9_120.npz"])
@pytest.mark.parametrize("lanes,eager,jpd,cheap_limit,free", [(16, 1, 20, 0, 0), (64, 1, 5, 3, 0), (32, 0, 20, 2, 8),
                                                              (3, 1, 5, 0, 1000)])
def test_shared_tt_helping_keeps_tricks(replay_lib, name, lanes, eager, jpd, cheap_limit, free):
    """Helpers search in their donor's TT: tricks stay the reference's, and every helper
    lets go of the donor's TT (the simulator returns -5 otherwise)."""
    g = load_golden(name)
    rc, t, st = block_shared(replay_lib, g["hands"][:48], lanes, eager, jpd, cheap_limit, free)
    assert rc == 0
    assert (t == g["tricks"][:48]).all()
    if eager:
        assert st[12] > 0


def test_shared_tt_helping_full_deals(replay_lib):
    g = load_golden("k13_24.npz")
    idx = [1, 3, 15]
    rc, t, st = block_shared(replay_lib, g["hands"][idx], 32, 1, 20, 3)
    assert rc == 0 and (t == g["tricks"][idx]).all() and st[12] > 0
