"""Test infrastructure: the learned guide's network restated in numpy (float64 arithmetic,
with the bf16 roundings the GPU kernels apply to weights, activations and gradients), the
CPU oracle the GPU forward and backward passes are checked against. Same parameter layout,
features and losses as dds_gpu_b200/csrc/ddg_guide.cuh."""
import numpy as np

IN, IN_PAD, HID, OUT_T, OUT_M, OUT_PAD, DO_LD = 217, 256, 256, 14, 52, 80, 128
OFF_W1 = 0
OFF_B1 = OFF_W1 + HID * IN_PAD
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + OUT_PAD * HID
N_PARAMS = OFF_B3 + OUT_PAD


def bf16(x):
    """Round to bfloat16 (nearest, ties to even), returned as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(HID, IN_PAD), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(HID, HID),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3].reshape(OUT_PAD, HID), p[OFF_B3:N_PARAMS])


def init_params(seed):
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, dtype=np.float32)
    a1, a2, a3 = np.sqrt(6 / (IN + HID)), np.sqrt(6 / (2 * HID)), np.sqrt(6 / (HID + OUT_T + OUT_M))
    w1 = np.zeros((HID, IN_PAD), np.float32)
    w1[:, :IN] = rng.uniform(-a1, a1, (HID, IN))
    w3 = np.zeros((OUT_PAD, HID), np.float32)
    w3[:OUT_T + OUT_M] = rng.uniform(-a3, a3, (OUT_T + OUT_M, HID))
    p[OFF_W1:OFF_B1] = w1.reshape(-1)
    p[OFF_W2:OFF_B2] = rng.uniform(-a2, a2, HID * HID)
    p[OFF_W3:OFF_B3] = w3.reshape(-1)
    return p


def card_bit(c):
    return (c // 13) * 16 + c % 13


def features(hands, rows):
    X = np.zeros((len(rows), IN_PAD))
    for i, e in enumerate(rows):
        if e < 0:
            continue
        deal, sd = e // 20, e % 20
        strain, decl = sd // 4, sd % 4
        leader = (decl + 1) & 3
        for seat in range(4):
            h = int(hands[deal, seat])
            for c in range(52):
                if (h >> card_bit(c)) & 1:
                    X[i, c * 4 + seat] = 1
        X[i, 208 + strain] = 1
        X[i, 213 + leader] = 1
    return X


def _gelu(z):
    from math import erf, sqrt
    v = np.vectorize(lambda t: 0.5 * t * (1 + erf(t / sqrt(2))))
    return v(z)


def _gelu_grad(z):
    from math import erf, exp, pi, sqrt
    v = np.vectorize(lambda t: 0.5 * (1 + erf(t / sqrt(2))) + t * exp(-0.5 * t * t) / sqrt(2 * pi))
    return v(z)


def loss_and_grads(params, hands, tricks20, best20, rows):
    """Mean loss over the batch (padded rows count in the mean, as on the GPU) and the
    gradients in the flat parameter layout."""
    W1, b1, W2, b2, W3, b3 = unpack(params)
    W1b, W2b, W3b = bf16(W1), bf16(W2), bf16(W3)
    B = len(rows)
    X = features(hands, rows)
    Z1 = X @ W1b.T + b1
    H1 = bf16(_gelu(Z1))
    Z2 = H1 @ W2b.T + b2
    H2 = bf16(_gelu(Z2))
    L = H2 @ W3b.T + b3
    dO = np.zeros((B, OUT_PAD))
    loss = 0.0
    for i, e in enumerate(rows):
        if e < 0:
            continue
        deal, sd = e // 20, e % 20
        decl = sd % 4
        leader = (decl + 1) & 3
        t = int(tricks20[deal, sd // 4, decl])
        if t > 13:
            continue
        ns = t if decl % 2 == 0 else 13 - t
        l = L[i, :OUT_T]
        p = np.exp(l - l.max())
        p /= p.sum()
        loss -= np.log(p[ns])
        g = p.copy()
        g[ns] -= 1
        dO[i, :OUT_T] = g
        best = int(best20[deal, sd // 4, decl])
        own = int(hands[deal, leader])
        if best >= 0 and (own >> best) & 1:
            y = (best >> 4) * 13 + (best & 15)
            mask = np.array([(own >> card_bit(c)) & 1 for c in range(52)], bool)
            lm = L[i, OUT_T:OUT_T + OUT_M]
            q = np.zeros(52)
            q[mask] = np.exp(lm[mask] - lm[mask].max())
            q /= q.sum()
            loss -= np.log(q[y])
            gq = q.copy()
            gq[y] -= 1
            dO[i, OUT_T:OUT_T + OUT_M] = np.where(mask, gq, 0)
    dO = bf16(dO / B)
    grad = np.zeros(N_PARAMS)
    grad[OFF_W3:OFF_B3] = (dO.T @ H2).reshape(-1)
    grad[OFF_B3:N_PARAMS] = dO.sum(0)
    dZ2 = bf16((dO @ W3b) * _gelu_grad(Z2))
    grad[OFF_W2:OFF_B2] = (dZ2.T @ H1).reshape(-1)
    grad[OFF_B2:OFF_W3] = dZ2.sum(0)
    dZ1 = bf16((dZ2 @ W2b) * _gelu_grad(Z1))
    grad[OFF_W1:OFF_B1] = (dZ1.T @ X).reshape(-1)
    grad[OFF_B1:OFF_W2] = dZ1.sum(0)
    return loss / B, grad, L
