"""CPU checks of the classifier oracle (oracle/mlp.py): its backprop against central finite
differences in float64-evaluated loss, and the bf16 rounding helper."""
import numpy as np

from oracle import mlp


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.0078125, -3.14159, 1e-3, 0.0], np.float32)
    r = mlp.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # ties to even
    assert r[2] == np.float32(1.0078125)
    assert abs(r[3] - -3.140625) < 1e-6
    assert (mlp.bf16(r) == r).all()


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    p = mlp.init_params(3)
    keys = rng.integers(0, 1 << 32, 64, dtype=np.uint64).astype(np.uint32)
    labels = (rng.random(64) < 0.25).astype(np.float32)
    _, g = mlp.loss_and_grads(p, keys, labels, 3.0, emulate=False)
    idx = np.concatenate([rng.choice(4096, 6, replace=False), 4096 + rng.choice(16384, 6, replace=False),
                          20480 + rng.choice(384, 6, replace=False), [20864]])
    for i in idx:
        h = 1e-4  # small: a ReLU kink inside [p-h, p+h] breaks the difference quotient
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mlp.loss_only(pp, keys, labels, 3.0) - mlp.loss_only(pm, keys, labels, 3.0)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-3 * abs(fd) + 2e-6, (i, fd, g[i])


def test_emulated_and_fp32_gradients_agree_to_bf16_precision():
    rng = np.random.default_rng(1)
    p = mlp.init_params(4)
    keys = rng.integers(0, 1 << 32, 512, dtype=np.uint64).astype(np.uint32)
    labels = (rng.random(512) < 0.1).astype(np.float32)
    _, g32 = mlp.loss_and_grads(p, keys, labels, 5.0, emulate=False)
    _, g16 = mlp.loss_and_grads(p, keys, labels, 5.0, emulate=True)
    assert np.linalg.norm(g16 - g32) / np.linalg.norm(g32) < 0.05
