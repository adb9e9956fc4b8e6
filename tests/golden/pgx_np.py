"""Pgx DDS result files (.npy, int32, shape (2, n, 4)) written and read with numpy (test
infrastructure). The layout is the dataset's, as the reference decodes it (src/npy.h:47-63)
and dd_gpu's FILE.npy mode reads it (dds_gpu_b200/csrc/npy_pgx.hpp):
  row 0, deal i, suit s (S,H,D,C): the 2-bit owner (N,E,S,W) of card k of the suit at
      shift 2*(12-k), cards in the order A,2,3,..,K;
  row 1, deal i, seat: the declarer's tricks in strain C,D,H,S,NT at shift 4*(4-strain).
Used to make small files of this project's own seeded deals and reference tables, so the
file mode is tested without copying any of the dataset's records.
"""
import numpy as np

_RANK_OF_K = [12] + list(range(12))  # card k of a suit's 13 (A first, then 2..K)


def encode(hands, tricks):
    """(n, 4) uint64 full 13-card deals and (n, 5, 4) tables -> (2, n, 4) int32 array."""
    hands = np.asarray(hands, dtype=np.uint64)
    tricks = np.asarray(tricks).reshape(-1, 5, 4)
    n = hands.shape[0]
    out = np.zeros((2, n, 4), dtype=np.int64)
    for s in range(4):
        for k, rank in enumerate(_RANK_OF_K):
            bit = np.uint64(1) << np.uint64(s * 16 + rank)
            owner = np.full(n, -1, dtype=np.int64)
            for seat in range(4):
                owner[(hands[:, seat] & bit) != 0] = seat
            if (owner < 0).any():
                raise ValueError("Pgx files hold full deals (every card dealt)")
            out[0, :, s] |= owner << (2 * (12 - k))
    for seat in range(4):
        for strain in range(5):
            out[1, :, seat] |= tricks[:, strain, seat].astype(np.int64) << (4 * (4 - strain))
    return out.astype(np.int32)


def decode(arr):
    """(2, n, 4) int32 -> hands (n, 4) uint64, tricks (n, 5, 4) uint8."""
    a = np.asarray(arr).astype(np.int64) & 0xFFFFFFFF
    n = a.shape[1]
    hands = np.zeros((n, 4), dtype=np.uint64)
    for s in range(4):
        for k, rank in enumerate(_RANK_OF_K):
            owner = (a[0, :, s] >> (2 * (12 - k))) & 3
            for seat in range(4):
                hands[owner == seat, seat] |= np.uint64(1) << np.uint64(s * 16 + rank)
    tricks = np.zeros((n, 5, 4), dtype=np.uint8)
    for seat in range(4):
        for strain in range(5):
            tricks[:, strain, seat] = (a[1, :, seat] >> (4 * (4 - strain))) & 15
    return hands, tricks


def write(path, hands, tricks):
    np.save(path, encode(hands, tricks))
