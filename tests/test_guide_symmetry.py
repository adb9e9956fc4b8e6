"""The guide's training augmentation (dds_gpu_b200.guide.augment) maps each deal to a
symmetric one: the oracle's tables of the transformed deals must equal the transformed
tables, and every transformed best lead must be a card of the new leader."""
import ctypes
import os

import numpy as np

from conftest import load_golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def oracle_tables(hands):
    import subprocess
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_build", "libddoracle.so"))
    lib.ddo_solve_batch.restype = ctypes.c_longlong
    P = ctypes.c_void_p
    lib.ddo_solve_batch.argtypes = [P, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P, P]
    h = np.ascontiguousarray(hands, dtype=np.uint64)
    out = np.zeros(h.shape[0] * 20, np.int32)
    assert lib.ddo_solve_batch(h.ctypes.data, h.shape[0], 10, 4, 5, None, out.ctypes.data, None) >= 0
    return out.reshape(-1, 5, 4)


def test_augment_keeps_double_dummy_results():
    from dds_gpu_b200.guide import augment
    g = load_golden("k5_120.npz")
    hands, tricks = g["hands"][:60], g["tricks"][:60]
    n = hands.shape[0]
    best = np.full((n, 5, 4), -1, np.int8)
    for d in range(n):  # some card of each leader as a stand-in lead label
        for decl in range(4):
            hh = int(hands[d, (decl + 1) & 3])
            best[d, :, decl] = hh.bit_length() - 1
    rng = np.random.default_rng(5)
    for _ in range(3):
        ah, at, ab = augment(hands, tricks, best, rng)
        assert (oracle_tables(ah) == at).all()
        for d in range(n):
            for st in range(5):
                for decl in range(4):
                    c = int(ab[d, st, decl])
                    assert c >= 0 and (int(ah[d, (decl + 1) & 3]) >> c) & 1
