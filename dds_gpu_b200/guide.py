"""The learned guide's pipeline: labels from the solver, training on the GPU (libddg's own
tensor-core forward/backward kernels), the weights file, and guided solves.

    python -m dds_gpu_b200.guide train [--deals N] [--seconds S] [--epochs E] [--out FILE]

Labels: seeded 13-card deals (seed 1000, never the benchmark's) solved by the plain solver
within a time budget; each finished (deal, strain, declarer) gives the NS trick count and
the lead that decided it (ddg_solve_device_ex's best leads). Jobs the budget did not reach
give no label, so the labels lean to the easier jobs. The weights file holds the fp32
parameters in ddg_guide's flat layout.
"""
import argparse
import os
import time

import numpy as np

from . import Guide, Solver, make_deals

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "guide_weights.npz")
TRAIN_SEED = 1000


def load_weights(path=WEIGHTS):
    """The trained parameters, or None when there is no weights file."""
    if not os.path.exists(path):
        return None
    with np.load(path) as z:
        return np.ascontiguousarray(z["params"], dtype=np.float32)


def init_params(seed):
    """Uniform (Glorot) initial weights, zero biases, zero padding rows and columns."""
    rng = np.random.default_rng(seed)
    n_in, hid, n_out, in_pad, out_pad = 217, 256, 66, 256, 80
    w1 = np.zeros((hid, in_pad), np.float32)
    w1[:, :n_in] = rng.uniform(-1, 1, (hid, n_in)) * np.sqrt(6 / (n_in + hid))
    w2 = (rng.uniform(-1, 1, (hid, hid)) * np.sqrt(6 / (2 * hid))).astype(np.float32)
    w3 = np.zeros((out_pad, hid), np.float32)
    w3[:n_out] = rng.uniform(-1, 1, (n_out, hid)) * np.sqrt(6 / (hid + n_out))
    return np.concatenate([w1.ravel(), np.zeros(hid, np.float32), w2.ravel(), np.zeros(hid, np.float32),
                           w3.ravel(), np.zeros(out_pad, np.float32)])


def label(solver, d_hands, n, torch):
    """Plain solve of n deals (device buffer) with best-lead output: (tricks u8 (n*20),
    best leads i8 (n*20)) as device tensors; unfinished entries are 255 / -1."""
    d_out = torch.empty(n * 20, dtype=torch.uint8, device=d_hands.device)
    d_best = torch.empty(n * 20, dtype=torch.int8, device=d_hands.device)
    st = solver.solve_device(d_hands.data_ptr(), n, d_out.data_ptr(), d_best=d_best.data_ptr())
    return d_out, d_best, st


def train(guide, d_hands, d_tricks, d_best, rows, epochs, batch=4096, lr=2e-3, seed=0, log=None):
    """Adam over shuffled example rows, cosine-decayed learning rate; returns the last
    epoch's mean loss and trick-head accuracy."""
    rng = np.random.default_rng(seed)
    steps = max(1, epochs * ((len(rows) + batch - 1) // batch))
    k = 0
    loss = acc = 0.0
    for ep in range(epochs):
        perm = rng.permutation(rows)
        tot_l = tot_h = tot_n = 0.0
        for i in range(0, len(perm), batch):
            part = perm[i:i + batch]
            a = lr * 0.5 * (1 + np.cos(np.pi * k / steps))
            l, h, c, _ = guide.step(d_hands.data_ptr(), d_tricks.data_ptr(), d_best.data_ptr(), part, a)
            tot_l += l * len(part)
            tot_h += h
            tot_n += c
            k += 1
        loss, acc = tot_l / len(perm), tot_h / max(1.0, tot_n)
        if log:
            log(f"epoch {ep + 1}/{epochs}: loss {loss:.4f}, trick-head accuracy {acc:.3f}")
    return loss, acc


def evaluate(guide, d_hands, n, d_tricks, torch):
    """Seed hit rate (exact / within one) on the labelled entries of n deals."""
    d_seed = torch.empty(n * 20, dtype=torch.int8, device=d_hands.device)
    guide.predict(d_hands.data_ptr(), n, d_seed.data_ptr(), 0)
    seeds = d_seed.cpu().numpy().reshape(n, 5, 4).astype(int)
    t = d_tricks.cpu().numpy().reshape(n, 5, 4).astype(int)
    ns = np.where(np.arange(4) % 2 == 0, t, 13 - t)
    ok = t <= 13
    return float((seeds == ns)[ok].mean()), float((abs(seeds - ns) <= 1)[ok].mean())


def main():
    import torch
    p = argparse.ArgumentParser()
    p.add_argument("cmd", choices=["train"])
    p.add_argument("--deals", type=int, default=20000)
    p.add_argument("--seconds", type=float, default=120.0, help="labelling budget")
    p.add_argument("--epochs", type=int, default=40)
    p.add_argument("--lr", type=float, default=2e-3)
    p.add_argument("--out", default=WEIGHTS)
    a = p.parse_args()
    hands = make_deals(TRAIN_SEED, 0, a.deals, 13)
    d_hands = torch.from_numpy(hands.view(np.int64)).cuda()
    solver = Solver(tt_log2=10, jobs_per_deal=5, time_limit_s=a.seconds)
    t0 = time.time()
    d_tricks, d_best, st = label(solver, d_hands, a.deals, torch)
    solver.close()
    t = d_tricks.cpu().numpy()
    labelled = np.nonzero(t <= 13)[0].astype(np.int64)
    print(f"labels: {len(labelled)} of {a.deals * 20} entries in {time.time() - t0:.0f} s "
          f"({st['nodes'] / 1e9:.1f} G nodes)", flush=True)
    # hold out the last tenth of the deals
    cut = (a.deals * 9 // 10) * 20
    tr, va = labelled[labelled < cut], labelled[labelled >= cut]
    guide = Guide(max_rows=4096, params=init_params(1))
    t1 = time.time()
    loss, acc = train(guide, d_hands, d_tricks, d_best, tr, a.epochs, lr=a.lr, log=lambda m: print(m, flush=True))
    print(f"trained in {time.time() - t1:.1f} s", flush=True)
    # held-out seed accuracy on the labelled validation entries
    vdeals = a.deals - a.deals * 9 // 10
    d_vh = d_hands[a.deals * 9 // 10:].contiguous()
    d_vt = d_tricks[cut:].contiguous()
    hit, near = evaluate(guide, d_vh, vdeals, d_vt, torch)
    print(f"held-out seeds: exact {hit:.3f}, within one {near:.3f} ({len(va)} labelled entries)", flush=True)
    params = guide.params()
    np.savez_compressed(a.out, params=params, train_seed=TRAIN_SEED, deals=a.deals, labels=len(tr),
                        epochs=a.epochs, holdout_exact=hit, holdout_within_one=near)
    print(f"wrote {a.out}", flush=True)
    guide.close()


if __name__ == "__main__":
    main()
