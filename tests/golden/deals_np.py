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


def _splitmix_int(x):
    x = (x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return x, z ^ (z >> 31)


def make_deals_mixed(seed, first, n, k_min=5, k_max=13, skew=0.3):
    """Uneven-hardness deals, restated in plain Python (small n only). Deal d: x = S ^
    (0x9E6C63D0676A9A99 * (d + 1)); K = k_min + next % (k_max - k_min + 1); skewed when
    (next >> 11) / 2^53 < skew; the 52 cards shuffled as in make_deals; a skewed deal then
    gives seat `lng` = next % 4 the first min(7 + next % 4, K) cards of suit `su` = next % 4
    (drawn in the order su, lng, void seat = (lng + 1 + next % 3) % 4, count) in shuffle
    order, the void seat its K cards of the other suits, and the rest go round-robin from
    seat 0 over the seats that still need cards (the void seat never takes suit su)."""
    M = 0xFFFFFFFFFFFFFFFF
    k_min, k_max = max(1, k_min), min(13, k_max)
    k_max = max(k_max, k_min)
    out = np.zeros((n, 4), dtype=np.uint64)
    for r in range(n):
        d = first + r
        x = (seed ^ ((0x9E6C63D0676A9A99 * (d + 1)) & M)) & M
        x, z = _splitmix_int(x)
        k = k_min + z % (k_max - k_min + 1)
        x, z = _splitmix_int(x)
        skewed = (z >> 11) * (1.0 / 9007199254740992.0) < skew
        cards = [(i // 13) * 16 + i % 13 for i in range(52)]
        for i in range(51, 0, -1):
            x, z = _splitmix_int(x)
            j = z % (i + 1)
            cards[i], cards[j] = cards[j], cards[i]
        h = [0, 0, 0, 0]
        cnt = [0, 0, 0, 0]
        su = lng = vd = -1
        if skewed:
            x, z = _splitmix_int(x)
            su = z % 4
            x, z = _splitmix_int(x)
            lng = z % 4
            x, z = _splitmix_int(x)
            vd = (lng + 1 + z % 3) % 4
            x, z = _splitmix_int(x)
            want = min(7 + z % 4, k)
            for i in range(52):
                if cnt[lng] >= want:
                    break
                if cards[i] >= 0 and cards[i] >> 4 == su:
                    h[lng] |= 1 << cards[i]
                    cnt[lng] += 1
                    cards[i] = -1
            for i in range(52):
                if cnt[vd] >= k:
                    break
                if cards[i] >= 0 and cards[i] >> 4 != su:
                    h[vd] |= 1 << cards[i]
                    cnt[vd] += 1
                    cards[i] = -1
        seat = 0
        for c in cards:
            if c < 0:
                continue
            for _ in range(4):
                if cnt[seat] < k and not (seat == vd and c >> 4 == su):
                    h[seat] |= 1 << c
                    cnt[seat] += 1
                    seat = (seat + 1) % 4
                    break
                seat = (seat + 1) % 4
            if min(cnt) >= k:
                break
        out[r] = h
    return out
