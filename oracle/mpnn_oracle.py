"""FP64 CPU restatement of the learned-initialisation network (the checker of
cudafusion_b200/csrc/cf_mpnn.cu).

TEST INFRASTRUCTURE ONLY: imported by tests/ and bench.py as the oracle; the
product library never loads it.  The reference has no such network (it starts
every frame's GN from a zero increment), so the oracle follows the network's
own definition:

    h1 = relu(W0 [x_i, mean_j x_j] + b0)      (20 + 20 -> 64)
    h2 = relu(W1 [h1_i, mean_j h1_j] + b1)    (64 + 64 -> 64)
    h3 = relu(W2 [h2_i, mean_j h2_j] + b2)    (64 + 64 -> 64)
    out = Wo h3_i + bo + x_i[0:6]             (64 -> 6)
    loss = mean over N*6 of (out - target)^2

With rounding=True every quantity the kernels keep in BF16 (parameters, the
network inputs, the activations h1..h3) is rounded to BF16 here too, and the
gradient treats the rounding as the identity, as the kernels do; sums run in
FP64.  `finite_differences` checks the analytic gradient of the unrounded
network.
"""
import numpy as np

IN, HID, OUT, K = 20, 64, 6, 8
SHAPES = [("W0", (HID, 2 * IN)), ("b0", (HID,)), ("W1", (HID, 2 * HID)), ("b1", (HID,)),
          ("W2", (HID, 2 * HID)), ("b2", (HID,)), ("Wo", (OUT, HID)), ("bo", (OUT,))]
PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16(x):
    """Round to BF16 (round to nearest even), returned as float64."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(theta):
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = np.asarray(theta[o:o + n], np.float64).reshape(shp)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SHAPES])


def graph(nbr):
    """Valid-neighbour mask and 1/degree (FP32, as the kernels hold it)."""
    nbr = np.asarray(nbr, np.int64)
    valid = nbr >= 0
    deg = valid.sum(1)
    inv = np.where(deg > 0, (1.0 / np.maximum(deg, 1)).astype(np.float32), np.float32(0)).astype(np.float64)
    return nbr, valid, inv


def _agg(h, nbr, valid, inv):
    idx = np.where(valid, nbr, 0)
    return (h[idx] * valid[..., None]).sum(1) * inv[:, None]


def forward(theta, x, nbr, rounding=True):
    r = bf16 if rounding else (lambda a: np.asarray(a, np.float64))
    P = {k: r(v) for k, v in unpack(theta).items()}
    nbr, valid, inv = graph(nbr)
    x = np.asarray(x, np.float64)
    cache = {"nbr": nbr, "valid": valid, "inv": inv, "P": P}
    h = r(x)
    layers = []
    for l in range(3):
        cat = np.concatenate([h, _agg(h, nbr, valid, inv)], 1)
        z = cat @ P[f"W{l}"].T + P[f"b{l}"]
        hn = r(np.maximum(z, 0.0))
        layers.append((cat, hn))
        h = hn
    out = h @ P["Wo"].T + P["bo"] + x[:, :OUT]
    cache["layers"] = layers
    cache["h3"] = h
    return out, cache


def loss_and_grad(theta, x, tgt, nbr, rounding=True):
    out, c = forward(theta, x, nbr, rounding)
    N = x.shape[0]
    d = out - np.asarray(tgt, np.float64)
    loss = float((d * d).sum() / (6.0 * N))
    dy = 2.0 * d / (6.0 * N)
    P, nbr, valid, inv = c["P"], c["nbr"], c["valid"], c["inv"]
    g = {"Wo": dy.T @ c["h3"], "bo": dy.sum(0)}
    dh = dy @ P["Wo"]
    for l in (2, 1, 0):
        cat, hn = c["layers"][l]
        dz = dh * (hn > 0)
        g[f"W{l}"] = dz.T @ cat
        g[f"b{l}"] = dz.sum(0)
        if l == 0:
            break
        dcat = dz @ P[f"W{l}"]
        din = HID
        dh = dcat[:, :din].copy()
        dagg = dcat[:, din:] * inv[:, None]
        idx = np.where(valid, nbr, 0)
        for k in range(K):
            np.add.at(dh, idx[valid[:, k], k], dagg[valid[:, k]])
    return loss, pack(g)


def finite_differences(theta, x, tgt, nbr, idx, eps=1e-6):
    """Central differences of the unrounded loss at parameter indices idx."""
    g = np.zeros(len(idx))
    for n, q in enumerate(idx):
        tp = np.array(theta, np.float64)
        tm = tp.copy()
        tp[q] += eps
        tm[q] -= eps
        g[n] = (loss_and_grad(tp, x, tgt, nbr, False)[0] - loss_and_grad(tm, x, tgt, nbr, False)[0]) / (2 * eps)
    return g
