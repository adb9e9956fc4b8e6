"""The learned guide: its tcgen05 forward and backward passes against the numpy oracle
(oracle/guide_ref.py), training on the GPU, and guided solves staying exact."""
import os
import sys

import numpy as np
import pytest

from conftest import load_golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import guide_ref  # noqa: E402

pytestmark = pytest.mark.gpu


def highest_leads(hands):
    """A lead label per example for the gradient check: the leader's highest card."""
    n = hands.shape[0]
    best = np.full((n, 5, 4), -1, np.int8)
    for d in range(n):
        for decl in range(4):
            h = int(hands[d, (decl + 1) & 3])
            if h:
                best[d, :, decl] = h.bit_length() - 1
    return best


def to_dev(a, dtype):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(dtype)).cuda()


def test_guide_gradients_match_oracle(ddg):
    import torch
    g = load_golden("k13_24.npz")
    hands, tricks = g["hands"], g["tricks"]
    best = highest_leads(hands)
    params = guide_ref.init_params(7)
    params[guide_ref.OFF_B1:guide_ref.OFF_W2] = 0.05  # non-zero biases exercise their paths
    params[guide_ref.OFF_B3:] = 0.01
    rows = np.arange(256, dtype=np.int64)
    rows[250:] = -1  # padded rows carry no example
    guide = ddg.Guide(max_rows=256, params=params)
    try:
        d_h, d_t, d_b = to_dev(hands, np.int64), to_dev(tricks.reshape(-1), np.uint8), to_dev(best.reshape(-1), np.int8)
        loss, hits, labelled, grad = guide.step(d_h.data_ptr(), d_t.data_ptr(), d_b.data_ptr(), rows, 0.0, True)
        torch.cuda.synchronize()
    finally:
        guide.close()
    ref_loss, ref_grad, _ = guide_ref.loss_and_grads(params, hands, tricks, best, rows)
    assert labelled == 250
    assert abs(loss - ref_loss) < 1e-3 * abs(ref_loss)
    parts = {"W1": (guide_ref.OFF_W1, guide_ref.OFF_B1), "b1": (guide_ref.OFF_B1, guide_ref.OFF_W2),
             "W2": (guide_ref.OFF_W2, guide_ref.OFF_B2), "b2": (guide_ref.OFF_B2, guide_ref.OFF_W3),
             "W3": (guide_ref.OFF_W3, guide_ref.OFF_B3), "b3": (guide_ref.OFF_B3, guide_ref.N_PARAMS)}
    for name, (a, b) in parts.items():
        r, x = ref_grad[a:b], grad[a:b].astype(np.float64)
        err = np.linalg.norm(x - r) / max(np.linalg.norm(r), 1e-12)
        assert err < 2e-2, (name, err)


def test_guide_trains_on_gpu_and_guided_solves_stay_exact(ddg):
    import torch
    g = load_golden("k13_24.npz")
    hands, tricks = g["hands"], g["tricks"]
    s = ddg.Solver(tt_log2=10, jobs_per_deal=5, lanes=4096, block=256, min_blocks=2)
    guide = ddg.Guide(max_rows=512, params=guide_ref.init_params(3))
    try:
        light = [1, 3, 15, 17, 22]
        h = np.ascontiguousarray(hands[light])
        n = len(light)
        d_h = to_dev(h, np.int64)
        d_out = torch.empty(n * 20, dtype=torch.uint8, device="cuda")
        d_best = torch.empty(n * 20, dtype=torch.int8, device="cuda")
        s.solve_device(d_h.data_ptr(), n, d_out.data_ptr(), d_best=d_best.data_ptr())
        assert (d_out.cpu().numpy().reshape(n, 5, 4) == tricks[light]).all()
        best = d_best.cpu().numpy()
        assert (best >= 0).mean() > 0.8  # most answers name the lead that decided them
        # the labelled leads are the leader's cards
        bh = best.reshape(n, 5, 4)
        for d in range(n):
            for st in range(5):
                for decl in range(4):
                    if bh[d, st, decl] >= 0:
                        assert (int(h[d, (decl + 1) & 3]) >> int(bh[d, st, decl])) & 1
        rows = np.arange(n * 20, dtype=np.int64)
        losses = []
        for _ in range(60):
            loss, hits, cnt, _ = guide.step(d_h.data_ptr(), d_out.data_ptr(), d_best.data_ptr(), rows, 3e-3)
            losses.append(loss)
        assert losses[-1] < 0.5 * losses[0]
        d_seed = torch.empty(n * 20, dtype=torch.int8, device="cuda")
        d_hint = torch.empty(n * 20, dtype=torch.int8, device="cuda")
        guide.predict(d_h.data_ptr(), n, d_seed.data_ptr(), d_hint.data_ptr())
        seeds = d_seed.cpu().numpy().reshape(n, 5, 4)
        ns = np.where(np.arange(4) % 2 == 0, tricks[light], 13 - tricks[light])
        assert (seeds == ns).mean() > 0.9  # it has learned these few tables
        d_out2 = torch.empty(n * 20, dtype=torch.uint8, device="cuda")
        st = s.solve_device(d_h.data_ptr(), n, d_out2.data_ptr(), d_seeds=d_seed.data_ptr(), d_hints=d_hint.data_ptr())
        assert (d_out2.cpu().numpy().reshape(n, 5, 4) == tricks[light]).all()
        assert st["jobs_done"] == n * 5
    finally:
        guide.close()
        s.close()


def test_trained_guide_saves_nodes(ddg):
    """The committed guide against the plain solver on fresh deals: the same tables, and
    fewer search nodes over the jobs both runs finished within the same time."""
    import torch
    import dds_gpu_b200.guide as ddg_guide
    params = ddg_guide.load_weights()
    if params is None:
        pytest.skip("no trained guide weights")
    n = 2000
    hands = ddg.make_deals(12345, 0, n, 13)
    d_h = to_dev(hands, np.int64)
    guide = ddg.Guide(max_rows=4096, params=params)
    d_seed = torch.empty(n * 20, dtype=torch.int8, device="cuda")
    d_hint = torch.empty(n * 20, dtype=torch.int8, device="cuda")
    guide.predict(d_h.data_ptr(), n, d_seed.data_ptr(), d_hint.data_ptr())
    guide.close()
    runs = []
    for guided in (False, True):
        s = ddg.Solver(tt_log2=10, jobs_per_deal=5, block=256, min_blocks=2, time_limit_s=12.0)
        try:
            d_out = torch.empty(n * 20, dtype=torch.uint8, device="cuda")
            d_nodes = torch.zeros(n * 5, dtype=torch.int64, device="cuda")
            s.solve_device(d_h.data_ptr(), n, d_out.data_ptr(), d_job_nodes=d_nodes.data_ptr(),
                           d_seeds=d_seed.data_ptr() if guided else 0, d_hints=d_hint.data_ptr() if guided else 0)
            runs.append((d_out.cpu().numpy().reshape(n, 5, 4), d_nodes.cpu().numpy()))
        finally:
            s.close()
    (t0, n0), (t1, n1) = runs
    both = (n0 > 0) & (n1 > 0)
    assert both.sum() > 1000
    fin = both.reshape(n, 5)
    assert (t0[fin] == t1[fin]).all()
    plain, guided = int(n0[both].sum()), int(n1[both].sum())
    print(f"guide: {both.sum()} jobs finished by both, nodes plain {plain}, guided {guided} "
          f"({guided / plain:.3f})")
    assert guided < plain
