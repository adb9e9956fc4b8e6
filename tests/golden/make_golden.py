"""Regenerates the golden fixtures of tests/golden/ from the reference solver itself
(oracle/_ref/libddref.so, built by oracle/build_ref.sh from the reference's headers).

    python tests/golden/make_golden.py          # all fixtures
    python tests/golden/make_golden.py mixed    # only the uneven-hardness one
    python tests/golden/make_golden.py sig      # only the signature-entry ones

Each fixture holds seeded deals (tests/golden/deals_np.py), the reference's trick tables
(dd_solve_strain, src/dd.h:926) and its search-node count per job, with one job per
(deal, strain) (jpd 5: the four leads share a TT) and per (deal, strain, declarer) (jpd 20,
the reference's stage machine, src/dd_wave.h:82-84), at the stated TT size.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
from deals_np import make_deals, make_deals_mixed  # noqa: E402

P = ctypes.c_void_p
REF = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libddref.so"))


def ref_solve(h, tt_log2=10, threads=8):
    n = h.shape[0]
    out = np.zeros(n * 20, np.int32)
    nodes = np.zeros(n * 5, np.uint64)
    rc = REF.ref_solve_batch(h.ctypes.data_as(P), ctypes.c_long(n), tt_log2, threads,
                             out.ctypes.data_as(P), nodes.ctypes.data_as(P))
    assert rc == 0
    return out.reshape(n, 5, 4).astype(np.uint8), nodes.astype(np.uint32)


def ref_wave20(h, tt_log2=10):
    n = h.shape[0]
    out = np.zeros(n * 20, np.int32)
    nodes = np.zeros(n * 20, np.uint64)
    rc = REF.ref_wave_batch(h.ctypes.data_as(P), ctypes.c_long(n), tt_log2, 20,
                            out.ctypes.data_as(P), nodes.ctypes.data_as(P), None)
    assert rc == 0
    return out.reshape(n, 5, 4).astype(np.uint8), nodes.astype(np.uint32)


def ref_guess(h, seeds, tt_log2=10, threads=8):
    n = h.shape[0]
    out = np.zeros(n * 20, np.int32)
    nodes = np.zeros(n * 5, np.uint64)
    s32 = np.ascontiguousarray(seeds.reshape(n * 20), dtype=np.int32)
    rc = REF.ref_solve_batch_guess(h.ctypes.data_as(P), ctypes.c_long(n), tt_log2, threads,
                                   s32.ctypes.data_as(P), out.ctypes.data_as(P), nodes.ctypes.data_as(P))
    assert rc == 0
    return out.reshape(n, 5, 4).astype(np.uint8), nodes.astype(np.uint32)


def fixture(name, seed, n, k, tt_log2=10, wave20=True):
    h = make_deals(seed, 0, n, k)
    t5, n5 = ref_solve(h, tt_log2)
    d = dict(seed=seed, k=k, tt_log2=tt_log2, hands=h, tricks=t5, nodes_jpd5=n5)
    if wave20:
        t20, n20 = ref_wave20(h, tt_log2)
        assert (t20 == t5).all()
        d["nodes_jpd20"] = n20
    np.savez_compressed(os.path.join(HERE, name), **d)
    print(name, n, "deals", int(n5.sum()), "nodes")
    return h, t5


def mixed_fixture(name, seed, n, k_min=5, k_max=13, skew=0.3, tt_log2=10):
    """Uneven-hardness deals (K ~ U{k_min..k_max}, a share `skew` with a 7-10 card suit
    facing a void), the workload of the persistent uneven batch."""
    h = make_deals_mixed(seed, 0, n, k_min, k_max, skew)
    t5, n5 = ref_solve(h, tt_log2)
    np.savez_compressed(os.path.join(HERE, name), seed=seed, k_min=k_min, k_max=k_max, skew=skew,
                        tt_log2=tt_log2, hands=h, tricks=t5, nodes_jpd5=n5)
    print(name, n, "deals", int(n5.sum()), "nodes")


def sig_fixtures():
    """The reference built with its 12-byte signature entries (-DDD_TT_SIG,
    oracle/_ref/libddref_sig.so): tricks and per-job nodes of endings and light full deals."""
    sig = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libddref_sig.so"))
    for name, h in (("sig_k6_120.npz", make_deals(106, 0, 120, 6)), ("sig_k9_120.npz", make_deals(109, 0, 120, 9)),
                    ("sig_k13_5.npz", make_deals(2, 0, 24, 13)[[1, 3, 15, 17, 22]])):
        h = np.ascontiguousarray(h)
        n = h.shape[0]
        out = np.zeros(n * 20, np.int32)
        nodes = np.zeros(n * 5, np.uint64)
        assert sig.ref_solve_batch(h.ctypes.data_as(P), ctypes.c_long(n), 10, 8, out.ctypes.data_as(P),
                                   nodes.ctypes.data_as(P)) == 0
        t = out.reshape(n, 5, 4).astype(np.uint8)
        exact, _ = ref_solve(h)
        assert (t == exact).all()  # no signature collision on these deals
        np.savez_compressed(os.path.join(HERE, name), tt_log2=10, hands=h, tricks=t, nodes_jpd5=nodes.astype(np.uint32))
        print(name, n, "deals", int(nodes.sum()), "nodes (signature entries)")


def main():
    only = sys.argv[1:]
    if only:  # regenerate the named fixtures only
        if "mixed" in only:
            mixed_fixture("mixed_300.npz", seed=3000, n=300)
        if "sig" in only:
            sig_fixtures()
        return
    # Config 1: K=6 endings, 4096 deals, TT_LOG2=10.
    fixture("k6_4096.npz", seed=1, n=4096, k=6)
    # Endings of every size the brute-force oracle and the search both cover.
    for k in range(1, 10):
        fixture(f"k{k}_120.npz", seed=100 + k, n=120, k=k)
    # Full deals: the first 24 deals of the 13-card benchmark set (seed 2).
    fixture("k13_24.npz", seed=2, n=24, k=13)
    # TT sizes.
    for tt in (9, 12):
        fixture(f"k7_200_tt{tt}.npz", seed=300 + tt, n=200, k=7, tt_log2=tt, wave20=False)
    # Seeded stepping search: seeds = true NS tricks + U{-2..2}, clamped by the solver.
    h = make_deals(400, 0, 200, 8)
    t, _ = ref_solve(h)
    ns = t.astype(np.int16).copy()
    ns[:, :, 1::2] = 13 - ns[:, :, 1::2]
    rng = np.random.default_rng(400)
    seeds = (ns + rng.integers(-2, 3, ns.shape)).astype(np.int8)
    tg, ng = ref_guess(h, seeds)
    assert (tg == t).all()
    np.savez_compressed(os.path.join(HERE, "k8_200_seeded.npz"), seed=400, k=8, tt_log2=10, hands=h,
                        seeds=seeds, tricks=tg, nodes_jpd5=ng)
    print("k8_200_seeded.npz", int(ng.sum()), "nodes")
    # Uneven-hardness deals, K = 5..13, 30 % skewed.
    mixed_fixture("mixed_300.npz", seed=3000, n=300)
    # The signature-entry build of the reference.
    sig_fixtures()


if __name__ == "__main__":
    main()
