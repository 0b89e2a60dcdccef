"""CPU: the FP64 restatement of the learned initialiser's network
(oracle/nn_oracle.py) against central finite differences of its own loss,
on a small batch with unrounded weights -- the check that pins the oracle
before it checks the library's BF16 training kernels."""
import numpy as np

from oracle import nn_oracle as N


def test_param_count():
    assert N.param_count() == 16 * 16 + 16 + 32 * 144 + 32 + 2 * (32 * 288 + 32) + 256 * 2304 + 256 + \
        128 * 256 + 128 + 3 * 128 + 3


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(4)
    B = 2
    params = np.concatenate([np.concatenate([rng.normal(0, np.sqrt(2.0 / i), o * i), rng.normal(0, 0.1, o)])
                             for o, i in N.LAYERS])
    x1 = rng.normal(size=(B, 256))
    x2 = rng.normal(size=(B, 256, 256))
    t = rng.normal(size=(B, 3))
    loss, grad, _ = N.forward_backward(params, x1, x2, t, bf16_weights=False)
    assert np.isfinite(loss)
    # a few parameters of every layer
    off = 0
    h = 1e-5
    for o, i in N.LAYERS:
        for q in rng.choice(o * i + o, size=3, replace=False):
            k = off + q
            p1, p2 = params.copy(), params.copy()
            p1[k] += h
            p2[k] -= h
            l1 = N.forward_backward(p1, x1, x2, t, bf16_weights=False)[0]
            l2 = N.forward_backward(p2, x1, x2, t, bf16_weights=False)[0]
            fd = (l1 - l2) / (2 * h)
            assert abs(fd - grad[k]) <= 1e-5 + 1e-4 * abs(fd), (o, i, q, fd, grad[k])
        off += o * i + o


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.0, 0.0], np.float32)
    r = N.bf16(x)
    assert r[0] == 1.0 and r[3] == -3.0 and r[4] == 0.0
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: to even (1.0)
    assert r[1] == 1.0
    assert r[2] == 1.0078125
