"""The learned preconditioner's CPU oracle: its backward pass against central
finite differences of its own forward pass (float64, bfloat16 rounding off)."""
import numpy as np
import pytest

from oracle import unet_oracle as U


@pytest.fixture
def exact():
    U.ROUND = False
    yield
    U.ROUND = True


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.001953125, 1.005859375, 1.01171875, -3.14159], np.float32)
    r = U.bf16(x)
    # 7-bit mantissa, ulp 2^-7 at 1: 1 + 2^-8 is a tie (to even: 1), 1 + 2^-9
    # rounds down, 1 + 3*2^-9 up, 1 + 3*2^-8 is a tie (to even: 1 + 2^-6)
    assert list(r[:5]) == [1.0, 1.0, 1.0, 1.0078125, 1.015625]
    assert r[5] == -3.140625


def test_backward_matches_finite_differences(exact):
    rng = np.random.default_rng(3)
    p = U.init_params(1)
    for k in p:
        if k.startswith("b"):
            p[k] = (rng.standard_normal(p[k].shape) * 0.1).astype(np.float32)
    r = rng.standard_normal((8, 8, 8)).astype(np.float32)
    target = rng.standard_normal((8, 8, 8))

    def loss(pp):
        _, c = U.forward(pp, r)
        return U.loss_grad(c["zn"], target)[0]

    _, c = U.forward(p, r)
    _, dz = U.loss_grad(c["zn"], target)
    g = U.backward(p, c, dz)
    h = 1e-4
    for name in ["W0a", "W1b", "W2b", "W3s", "W4a", "W4b", "W5", "b3a", "b4b", "b0b"]:
        flat = p[name].reshape(-1)
        for idx in rng.choice(flat.size, 3, replace=False):
            q = {k: v.astype(np.float64).copy() for k, v in p.items()}
            q[name].reshape(-1)[idx] += h
            lp = loss(q)
            q[name].reshape(-1)[idx] -= 2 * h
            lm = loss(q)
            fd = (lp - lm) / (2 * h)
            an = g[name].reshape(-1)[idx]
            assert abs(fd - an) <= 1e-5 + 1e-4 * abs(fd), (name, idx, fd, an)
