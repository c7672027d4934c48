"""The warm-start U-Net's GPU kernels against the CPU oracle.

Forward outputs within 1e-5 relative L2 of the oracle (the GPU sums in
FP32, the oracle in float64, both with the same BF16-rounded weights) and
parameter gradients within 1e-4; training steps lower the loss and are
deterministic."""
import numpy as np
import pytest

from conftest import rel
from oracle import unet_oracle as U

pytestmark = pytest.mark.gpu


def _net(H, n):
    from sparseimaging_b200 import warmstart
    return warmstart.UNet(H, H, n)


def test_unet_forward_and_gradient_match_oracle(gpulib):
    rng = np.random.default_rng(3)
    net = _net(16, 2)
    p = net.params()  # the library's He initialisation
    lay, hw, hb, n = U.layout()
    p[hw:] = np.abs(p[hw:])  # a head with positive output where the features are
    p[-1] = 0.05
    net.set_params(p)
    x = rng.standard_normal((2, 2, 16, 16)).astype(np.float32)
    t = np.abs(rng.standard_normal((2, 16, 16))).astype(np.float32)
    o = U.UNetOracle(p)
    y_ref = o.forward(x)
    assert rel(net.forward(x), y_ref) < 1e-5
    loss, g = net.grad(x, t)
    loss_ref, g_ref = o.loss_and_grad(x, t)
    assert abs(loss - loss_ref) <= 1e-5 * loss_ref
    assert rel(g, g_ref) < 1e-4
    for w0, b0 in lay:  # every layer's block, not just the whole vector
        assert rel(g[w0:b0], g_ref[w0:b0]) < 1e-3
    net.close()


def test_unet_training_lowers_the_loss_deterministically(gpulib):
    rng = np.random.default_rng(4)
    x = rng.standard_normal((4, 2, 32, 32)).astype(np.float32)
    t = np.maximum(x[:, 0] * 0.5 + 0.1, 0).astype(np.float32)  # a learnable map of the input
    runs = []
    for _ in range(2):
        net = _net(32, 4)
        first = net.train_step(x, t, 3e-3)
        for _ in range(150):
            last = net.train_step(x, t, 3e-3)
        assert last < 0.3 * first
        runs.append(net.params())
        net.close()
    assert np.array_equal(runs[0], runs[1])


def test_unet_rejects_bad_shapes(gpulib):
    from sparseimaging_b200 import warmstart
    with pytest.raises(gpulib.MfistaError):
        warmstart.UNet(20, 20, 2)  # not a multiple of 8
    net = _net(16, 2)
    x = np.zeros((3, 2, 16, 16), np.float32)
    out = np.zeros((3, 16, 16), np.float32)
    L = warmstart._lib()
    assert L.mfista_unet_forward(net.h, warmstart._fp(x), 3, warmstart._fp(out)) == 2  # batch above its maximum
    assert L.mfista_unet_forward(net.h, warmstart._fp(x), 0, warmstart._fp(out)) == 2
    net.close()
