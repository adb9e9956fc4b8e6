"""The oracle (oracle/dd_oracle.c, a plain-C restatement of the reference's solve) pinned
against: the reference's own golden tables and node counts (tests/golden), an unpruned
minimax on small endings, the reference compiled here (oracle/_ref, when built) on fresh
deals, and the Pgx DDS tables shipped with the reference (read in place, when present)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden
from deals_np import make_deals

P = ctypes.c_void_p
ORACLE_DIR = os.path.join(ROOT, "oracle")
REF_SO = os.path.join(ORACLE_DIR, "_ref", "libddref.so")
# The reference tree, as the recipe that compiles it resolves it (REF_DIR or its default).
REF_DIR = subprocess.run(["bash", os.path.join(ORACLE_DIR, "build_ref.sh"), "--where"], capture_output=True,
                         text=True).stdout.strip()
PGX = os.path.join(REF_DIR, "data", "deals_20k.npy")


@pytest.fixture(scope="session")
def oracle():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    lib = ctypes.CDLL(os.path.join(ORACLE_DIR, "_build", "libddoracle.so"))
    lib.ddo_solve_batch.restype = ctypes.c_longlong
    lib.ddo_solve_batch.argtypes = [P, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P]
    lib.ddo_brute.argtypes = [P, ctypes.c_int, ctypes.c_int]
    return lib


def osolve(lib, hands, tt_log2=10, jpd=5, seeds=None, threads=8):
    n = hands.shape[0]
    h = np.ascontiguousarray(hands, dtype=np.uint64)
    out = np.zeros(n * 20, np.int32)
    nodes = np.zeros(n * jpd, np.uint64)
    sd = None if seeds is None else np.ascontiguousarray(seeds, dtype=np.int8).reshape(-1)
    total = lib.ddo_solve_batch(h.ctypes.data, n, tt_log2, threads, jpd, None if sd is None else sd.ctypes.data,
                                out.ctypes.data, nodes.ctypes.data)
    assert total == int(nodes.sum())
    return out.reshape(n, 5, 4), nodes


@pytest.mark.parametrize("name", [f"k{k}_120.npz" for k in range(1, 10)] + ["k6_4096.npz"])
@pytest.mark.parametrize("jpd", [5, 20])
def test_oracle_vs_reference_golden(oracle, name, jpd):
    g = load_golden(name)
    t, nodes = osolve(oracle, g["hands"], int(g["tt_log2"]), jpd)
    assert (t == g["tricks"]).all()
    assert (nodes == g[f"nodes_jpd{jpd}"]).all()


def test_oracle_full_deals(oracle):
    g = load_golden("k13_24.npz")
    t, nodes = osolve(oracle, g["hands"][:12])
    assert (t == g["tricks"][:12]).all() and (nodes == g["nodes_jpd5"][:60]).all()


@pytest.mark.parametrize("tt", [9, 12])
def test_oracle_tt_sizes(oracle, tt):
    g = load_golden(f"k7_200_tt{tt}.npz")
    t, nodes = osolve(oracle, g["hands"], tt)
    assert (t == g["tricks"]).all() and (nodes == g["nodes_jpd5"]).all()


def test_oracle_seeded(oracle):
    g = load_golden("k8_200_seeded.npz")
    t, nodes = osolve(oracle, g["hands"], 10, 5, g["seeds"])
    assert (t == g["tricks"]).all() and (nodes == g["nodes_jpd5"]).all()


@pytest.mark.parametrize("k", [1, 2, 3, 4])
def test_oracle_vs_minimax(oracle, k):
    """Known answers of an unpruned minimax (the reference's tests/test_small.cpp check):
    every strain and every leader; the solver's table gives NS tricks for leader d+1."""
    h = make_deals(500 + k, 0, 60, k)
    t, _ = osolve(oracle, h)
    for i in range(h.shape[0]):
        hi = np.ascontiguousarray(h[i])
        for strain in range(5):
            for decl in range(4):
                ns = oracle.ddo_brute(hi.ctypes.data, strain, (decl + 1) & 3)
                want = ns if decl % 2 == 0 else 13 - ns
                assert t[i, strain, decl] == want


def test_oracle_vs_reference_build(oracle):
    """Fresh deals against the reference compiled from its sources (when built here)."""
    if not os.path.exists(REF_SO):
        pytest.skip("oracle/_ref not built (reference sources absent)")
    ref = ctypes.CDLL(REF_SO)
    for k, n, seed in [(5, 400, 9001), (8, 150, 9002), (10, 30, 9003)]:
        h = make_deals(seed, 0, n, k)
        out = np.zeros(n * 20, np.int32)
        nodes = np.zeros(n * 5, np.uint64)
        assert ref.ref_solve_batch(h.ctypes.data_as(P), ctypes.c_long(n), 10, 8, out.ctypes.data_as(P),
                                   nodes.ctypes.data_as(P)) == 0
        t, mine = osolve(oracle, h)
        assert (t.reshape(-1) == out).all() and (mine == nodes).all()


def test_oracle_vs_pgx_tables(oracle):
    """Pgx DDS tables shipped with the reference (data/deals_20k.npy, read in place): 13 of
    its first 16 deals (the three slowest left out to keep the CPU suite short). Tricks do
    not depend on the TT size, so a larger TT is used."""
    if not (os.path.exists(PGX) and os.path.exists(REF_SO)):
        pytest.skip("reference data or shim absent")
    ref = ctypes.CDLL(REF_SO)
    n = 16
    hands = np.zeros((n, 4), np.uint64)
    want = np.zeros(n * 20, np.int32)
    assert ref.ref_pgx_load(PGX.encode(), ctypes.c_long(0), ctypes.c_long(n), hands.ctypes.data_as(P),
                            want.ctypes.data_as(P)) == 0
    keep = [i for i in range(n) if i not in (2, 3, 12)]
    t, _ = osolve(oracle, hands[keep], tt_log2=16)
    assert (t.reshape(len(keep), 20) == want.reshape(n, 20)[keep]).all()
