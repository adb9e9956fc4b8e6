"""Numpy restatement of the seeded deal generator (test infrastructure).

Deal d of seed S: x = S ^ (0xD1B54A32D192ED03 * (d + 1)); splitmix64 steps of x drive a
Fisher-Yates shuffle (i = 51..1, j = next % (i + 1)) of the cards (i // 13) * 16 + i % 13;
shuffle positions 0..4k-1 go round-robin to N, E, S, W. The product's C generator
(ddg_make_deals) must give the same bytes; tests/test_deals.py checks that.
"""
import numpy as np

_U = np.uint64


def _splitmix(x):
    x = x + _U(0x9E3779B97F4A7C15)
    z = x
    z = (z ^ (z >> _U(30))) * _U(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> _U(27))) * _U(0x94D049BB133111EB)
    return x, z ^ (z >> _U(31))


def make_deals(seed, first, n, k=13):
    with np.errstate(over="ignore"):
        d = np.arange(first, first + n, dtype=np.uint64)
        x = _U(seed) ^ (_U(0xD1B54A32D192ED03) * (d + _U(1)))
        base = np.array([(i // 13) * 16 + i % 13 for i in range(52)], dtype=np.int64)
        cards = np.tile(base, (n, 1))
        rows = np.arange(n)
        for i in range(51, 0, -1):
            x, z = _splitmix(x)
            j = (z % _U(i + 1)).astype(np.int64)
            a = cards[rows, i].copy()
            cards[rows, i] = cards[rows, j]
            cards[rows, j] = a
        hands = np.zeros((n, 4), dtype=np.uint64)
        for p in range(4 * k):
            hands[:, p % 4] |= _U(1) << cards[:, p].astype(np.uint64)
    return hands
