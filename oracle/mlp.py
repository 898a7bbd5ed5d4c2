"""CPU reference of the learned split's classifier — TEST INFRASTRUCTURE ONLY.

MLP 32 -> 128 -> 128 -> 1 over x_i = +1/-1 for bit i of the key, ReLU hidden layers, weighted
binary cross-entropy (mean over the batch).  Flat fp32 parameter layout:
W1[128x32] | W2[128x128] | b1[128] | b2[128] | w3[128] | b3.

`emulate=True` rounds where the GPU kernels (qsketch_b200/csrc/qs_mlp.cu) store bf16: the two
weight matrices, h1, h2, dh2 and dh1; sums stay fp32.  `emulate=False` is plain fp32 throughout.
There is no reference implementation of this part (the learned split has no counterpart in
the reference); the backprop itself is checked against central finite differences.
"""
import numpy as np

N_PARAMS = 4096 + 16384 + 128 + 128 + 128 + 1


def bf16(x):
    """Round float32 to bfloat16 (round to nearest even), returned as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(np.shape(x))


def unpack(p):
    p = np.asarray(p, np.float32)
    W1 = p[:4096].reshape(128, 32)
    W2 = p[4096:20480].reshape(128, 128)
    b1, b2, w3 = p[20480:20608], p[20608:20736], p[20736:20864]
    return W1, W2, b1, b2, w3, p[20864]


def features(keys):
    k = np.asarray(keys, np.uint32)[:, None]
    return (((k >> np.arange(32, dtype=np.uint32)) & 1).astype(np.float32) * 2.0 - 1.0)


def forward(p, keys, emulate=True):
    W1, W2, b1, b2, w3, b3 = unpack(p)
    if emulate:
        W1, W2 = bf16(W1), bf16(W2)
    X = features(keys)
    h1 = np.maximum(X @ W1.T + b1, 0.0).astype(np.float32)
    if emulate:
        h1 = bf16(h1)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0).astype(np.float32)
    if emulate:
        h2 = bf16(h2)
    z = (h2 @ w3 + b3).astype(np.float32)
    return z, (X, h1, h2, W2)


def loss_and_grads(p, keys, labels, pos_weight, emulate=True):
    z, (X, h1, h2, W2) = forward(p, keys, emulate)
    _, _, _, _, w3, _ = unpack(p)
    y = np.asarray(labels, np.float32)
    w = np.where(y > 0, np.float32(pos_weight), np.float32(1.0))
    n = z.size
    loss = float(np.mean(w * (np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))))
    dz = ((1.0 / (1.0 + np.exp(-z)) - y) * w / n).astype(np.float32)
    g3 = h2.T @ dz
    gb3 = np.float32(dz.sum())
    dh2 = np.where(h2 > 0, dz[:, None] * w3[None, :], 0.0).astype(np.float32)
    if emulate:
        dh2 = bf16(dh2)
    gW2 = dh2.T @ h1
    gb2 = dh2.sum(0)
    dh1 = np.where(h1 > 0, dh2 @ W2, 0.0).astype(np.float32)
    if emulate:
        dh1 = bf16(dh1)
    gW1 = dh1.T @ X
    gb1 = dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gW2.ravel(), gb1, gb2, g3, [gb3]]).astype(np.float32)
    return loss, g


def loss_only(p, keys, labels, pos_weight):
    """The loss in float64 throughout (for finite differences)."""
    W1, W2, b1, b2, w3, b3 = (np.asarray(a, np.float64) for a in unpack(p))
    X = features(keys).astype(np.float64)
    h2 = np.maximum(np.maximum(X @ W1.T + b1, 0.0) @ W2.T + b2, 0.0)
    z = h2 @ w3 + b3
    y = np.asarray(labels, np.float64)
    w = np.where(y > 0, pos_weight, 1.0)
    return float(np.mean(w * (np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))))


def init_params(seed):
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    p[:4096] = rng.uniform(-np.sqrt(6 / 32), np.sqrt(6 / 32), 4096)
    p[4096:20480] = rng.uniform(-np.sqrt(6 / 128), np.sqrt(6 / 128), 16384)
    p[20480:20864] = rng.uniform(-0.1, 0.1, 384)
    p[20736:20864] = rng.uniform(-np.sqrt(6 / 129), np.sqrt(6 / 129), 128)
    return p
