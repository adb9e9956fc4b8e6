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


def augment(hands, tricks, best, rng):
    """A random symmetry of each deal that keeps double-dummy results: a permutation of
    the four suits (the strain follows its trump suit; no trump stays) and a rotation of
    the seats (declarer d of the new deal is declarer d + r of the old one, so the
    declarer's trick count and best lead carry over). hands (n, 4) uint64, tricks and
    best (n, 5, 4); returns the three transformed arrays."""
    n = hands.shape[0]
    perm = np.argsort(rng.random((n, 4)), axis=1)           # suit s -> perm[:, s]
    rot = rng.integers(0, 4, n)
    h = hands.astype(np.uint64)
    moved = np.zeros_like(h)
    for s in range(4):
        part = (h >> np.uint64(16 * s)) & np.uint64(0x1FFF)
        moved |= part << (np.uint64(16) * perm[:, s].astype(np.uint64))[:, None]
    idx = (np.arange(4)[None, :] + rot[:, None]) % 4         # new seat s' <- old seat s' + r
    rows = np.arange(n)[:, None]
    new_hands = moved[rows, idx]
    # strain st (trump suit 3 - st) -> 3 - perm[3 - st]; no trump stays
    smap = np.empty((n, 5), np.int64)
    for st in range(4):
        smap[:, st] = 3 - perm[np.arange(n), 3 - st]
    smap[:, 4] = 4
    new_tricks = np.empty_like(tricks)
    new_best = np.empty_like(best)
    b = best.astype(np.int64)
    bsuit = np.where(b >= 0, b >> 4, 0)
    bmapped = np.where(b >= 0, perm[np.arange(n)[:, None, None], bsuit] * 16 + (b & 15), -1)
    # Tables hold the declarer's side's tricks as NS for N/S and 13 - NS for E/W (also for
    # fewer than 13 cards): go through NS tricks, which an odd rotation hands to the pair
    # that was EW (k - NS with k cards per hand).
    k = np.array([bin(int(x)).count("1") for x in hands[:, 0]], np.int64)[:, None]
    odd = (rot % 2 == 1)[:, None]
    even_decl = (np.arange(4) % 2 == 0)[None, :]
    for st in range(5):
        dst = smap[:, st]
        src_t = tricks[rows, st, idx].astype(np.int64)         # (n, 4): new declarer d' <- old d' + r
        src_even = ((np.arange(4)[None, :] + rot[:, None]) % 2) == 0
        ns_old = np.where(src_even, src_t, 13 - src_t)
        ns_new = np.where(odd, k - ns_old, ns_old)
        t_new = np.where(even_decl, ns_new, 13 - ns_new)
        t_new = np.where(src_t > 13, src_t, t_new)             # unsolved entries stay unsolved
        new_tricks[np.arange(n), dst] = t_new.astype(tricks.dtype)
        new_best[np.arange(n), dst] = bmapped[rows, st, idx]
    return new_hands, new_tricks, new_best.astype(np.int8)


def train(guide, d_hands, d_tricks, d_best, rows, epochs, batch=4096, lr=2e-3, seed=0, log=None,
          augment_from=None):
    """Adam over shuffled example rows, cosine-decayed learning rate; returns the last
    epoch's mean loss and trick-head accuracy."""
    rng = np.random.default_rng(seed)
    steps = max(1, epochs * ((len(rows) + batch - 1) // batch))
    k = 0
    loss = acc = 0.0
    for ep in range(epochs):
        if augment_from is not None and ep > 0:
            # a fresh symmetry of every training deal each epoch (the first epoch sees them as dealt)
            hands, tricks, best, torch = augment_from
            ah, at, ab = augment(hands, tricks, best, rng)
            d_hands.copy_(torch.from_numpy(ah.view(np.int64)))
            d_tricks.copy_(torch.from_numpy(np.ascontiguousarray(at).reshape(-1)))
            d_best.copy_(torch.from_numpy(np.ascontiguousarray(ab).reshape(-1)))
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
    p.add_argument("--augment", type=int, default=1, help="1: a random suit permutation and seat rotation "
                   "of every training deal each epoch")
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
    # hold out the last tenth of the deals; train on copies of the rest (augmented per epoch)
    ntr = a.deals * 9 // 10
    cut = ntr * 20
    tr, va = labelled[labelled < cut], labelled[labelled >= cut]
    th = np.ascontiguousarray(hands[:ntr])
    tt = d_tricks[:cut].cpu().numpy().reshape(ntr, 5, 4)
    tb = d_best[:cut].cpu().numpy().reshape(ntr, 5, 4)
    d_th = torch.from_numpy(th.view(np.int64)).cuda()
    d_tt = d_tricks[:cut].clone()
    d_tb = d_best[:cut].clone()
    # with augmentation every entry of a labelled deal may carry a label after a symmetry
    rows = np.arange(cut, dtype=np.int64) if a.augment else tr
    guide = Guide(max_rows=4096, params=init_params(1))
    t1 = time.time()
    loss, acc = train(guide, d_th, d_tt, d_tb, rows, a.epochs, lr=a.lr, log=lambda m: print(m, flush=True),
                      augment_from=(th, tt, tb, torch) if a.augment else None)
    print(f"trained in {time.time() - t1:.1f} s", flush=True)
    # held-out seed accuracy on the labelled validation entries
    vdeals = a.deals - a.deals * 9 // 10
    d_vh = d_hands[a.deals * 9 // 10:].contiguous()
    d_vt = d_tricks[cut:].contiguous()
    hit, near = evaluate(guide, d_vh, vdeals, d_vt, torch)
    print(f"held-out seeds: exact {hit:.3f}, within one {near:.3f} ({len(va)} labelled entries)", flush=True)
    params = guide.params()
    np.savez_compressed(a.out, params=params, train_seed=TRAIN_SEED, deals=a.deals, labels=len(tr),
                        epochs=a.epochs, augment=a.augment, holdout_exact=hit, holdout_within_one=near)
    print(f"wrote {a.out}", flush=True)
    guide.close()


if __name__ == "__main__":
    main()
