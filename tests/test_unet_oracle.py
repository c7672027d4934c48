"""The warm-start U-Net oracle against finite differences (CPU).

The oracle is the checker of the GPU network's gradients, so it is pinned
here by central differences of its own loss (float64 weights)."""
import numpy as np

from oracle import unet_oracle as U


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    lay, hw, hb, n = U.layout()
    p = rng.standard_normal(n) * 0.15
    x = rng.standard_normal((1, 2, 16, 16))
    t = np.abs(rng.standard_normal((1, 16, 16)))
    loss, g = U.UNetOracle(p, round_bf16=False).loss_and_grad(x, t)
    assert loss > 0
    # a spread of parameters: first/last conv weights, a bias, the head
    for k in [0, 5, lay[0][1], lay[8][0] + 3, lay[16][0] + 7, hw + 2, hb]:
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        lp, _ = U.UNetOracle(pp, round_bf16=False).loss_and_grad(x, t)
        lm, _ = U.UNetOracle(pm, round_bf16=False).loss_and_grad(x, t)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * max(abs(fd), 1e-6), (k, fd, g[k])


def test_layout_size():
    lay, hw, hb, n = U.layout()
    assert n == hb + 1 and hw + 16 == hb
    assert lay[0] == (0, 16 * 2 * 9)


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.14159], np.float32)
    r = U.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0   # halfway (1 + 2^-8) rounds to even
    assert r[2] == 1.0078125              # above halfway rounds up
    assert abs(r[3] + 3.140625) < 1e-12
