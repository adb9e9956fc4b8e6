"""Host-side pieces that need no GPU: the uneven-hardness deal generator and the guide's
parameter layout shared by the library, the training script and the numpy oracle."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def suit_len(h, s):
    return bin((int(h) >> (16 * s)) & 0x1FFF).count("1")


def test_mixed_deals_are_valid_and_uneven(ddg):
    hands = ddg.make_deals_mixed(7, 0, 4000, 5, 13, 0.3)
    assert all(ddg.check_deal(h) for h in hands)
    ks = np.array([bin(int(h[0])).count("1") for h in hands])
    assert ks.min() == 5 and ks.max() == 13
    assert all((np.bincount(ks)[5:] > 300))  # every K from 5 to 13 is drawn
    skewed = 0
    for h, k in zip(hands, ks):
        for s in range(4):
            lens = [suit_len(h[i], s) for i in range(4)]
            if max(lens) >= min(7, k) and min(lens) == 0:
                skewed += 1
                break
    assert 0.25 < skewed / len(hands) < 0.45  # the 30 % skewed, plus voids that occur anyway
    # the same seed and range give the same deals; ranges can be made alone
    again = ddg.make_deals_mixed(7, 1000, 10, 5, 13, 0.3)
    assert (again == hands[1000:1010]).all()


def test_guide_parameter_layout_agrees(ddg):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import guide_ref
    from dds_gpu_b200 import guide
    n = ddg.Guide.param_count()
    assert n == guide_ref.N_PARAMS == guide.init_params(1).size
    p = guide.init_params(3)
    w1 = p[guide_ref.OFF_W1:guide_ref.OFF_B1].reshape(256, 256)
    w3 = p[guide_ref.OFF_W3:guide_ref.OFF_B3].reshape(80, 256)
    assert not w1[:, 217:].any() and not w3[66:].any()  # padding stays zero
    assert not p[guide_ref.OFF_B1:guide_ref.OFF_W2].any()
    weights = guide.load_weights()
    if weights is not None:
        assert weights.size == n and np.isfinite(weights).all()
