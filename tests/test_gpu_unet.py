"""The warm-start U-Net's GPU kernels against the CPU oracle.

Forward outputs within 1e-5 relative L2 of the oracle (the GPU convolves on
the tensor cores with BF16 weights and the activations split into two BF16
planes, accumulating in FP32; the oracle in float64, both with the same
BF16-rounded weights) and parameter gradients within 1e-4; training steps
lower the loss and are deterministic."""
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


def test_tensor_core_convolutions_match_cuda_core_ones(gpulib, monkeypatch):
    """The tensor-core convolutions (default) and the FP32 CUDA-core ones
    (MFISTA_UNET_CUDA_CORES=1) give the same network output to 1e-5 on a
    64 x 64 batch, every level and both channel widths of the kernel, and
    the same parameter gradients to 5e-4: the tensor-core operands carry 16
    significant bits (BF16 hi/lo planes), and the weight gradients sum 4096
    strongly cancelling products per tile over the batch (measured 1.3e-4)."""
    rng = np.random.default_rng(5)
    x = rng.standard_normal((3, 2, 64, 64)).astype(np.float32)
    outs = []
    for cc in ("0", "1"):
        monkeypatch.setenv("MFISTA_UNET_CUDA_CORES", cc)
        net = _net(64, 3)
        p = net.params()
        lay, hw, hb, n = U.layout()
        p[hw:] = np.abs(p[hw:])
        net.set_params(p)
        outs.append(net.forward(x))
        _, g = net.grad(x, np.abs(x[:, 0]))
        outs.append(g)
        net.close()
    assert rel(outs[0], outs[2]) < 1e-5
    assert rel(outs[1], outs[3]) < 5e-4
