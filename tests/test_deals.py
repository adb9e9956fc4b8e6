"""Seeded deals: the product's C generator against the numpy restatement, and deal checks."""
import numpy as np

from deals_np import make_deals as np_deals


def test_generator_matches_restatement(ddg):
    for k in (1, 6, 13):
        a = ddg.make_deals(12345, 0, 300, k)
        b = np_deals(12345, 0, 300, k)
        assert (a == b).all()


def test_mixed_generator_matches_restatement(ddg):
    from deals_np import make_deals_mixed
    for seed, first, n, kmin, kmax, skew in ((3000, 0, 300, 5, 13, 0.3), (7, 500, 100, 7, 10, 0.6),
                                             (1, 0, 50, 13, 13, 1.0)):
        a = ddg.make_deals_mixed(seed, first, n, kmin, kmax, skew)
        b = make_deals_mixed(seed, first, n, kmin, kmax, skew)
        assert (a == b).all()


def test_generator_random_access(ddg):
    whole = ddg.make_deals(7, 0, 50, 13)
    part = ddg.make_deals(7, 20, 10, 13)
    assert (whole[20:30] == part).all()


def test_deals_are_valid(ddg):
    h = ddg.make_deals(99, 0, 200, 13)
    assert all(ddg.check_deal(x) for x in h)
    for x in h:
        assert int(x[0]) | int(x[1]) | int(x[2]) | int(x[3]) == 0x1FFF1FFF1FFF1FFF
    e = ddg.make_deals(99, 0, 20, 6)
    assert all(bin(int(v)).count("1") == 6 for v in e.ravel())


def test_check_deal_rejects_bad_deals(ddg):
    h = ddg.make_deals(1, 0, 1, 5)[0].copy()
    bad = h.copy()
    low = int(bad[0]) & -int(bad[0])
    bad[1] |= np.uint64(low)  # a card held twice
    assert not ddg.check_deal(bad)
    bad = h.copy()
    bad[2] = 0
    assert not ddg.check_deal(bad)  # unequal sizes
    bad = h.copy()
    bad[0] |= np.uint64(1) << np.uint64(13)  # rank 13 does not exist
    assert not ddg.check_deal(bad)
    assert not ddg.check_deal(np.zeros(4, np.uint64))  # empty hands
