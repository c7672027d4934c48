"""Learned warm start at the config-4 scale (256 x 256, M = 19998 shared
coverage): the committed network (sparseimaging_b200/data/unet_warmstart_256.npy,
trained by warmstart.config4_main on 1024 skies) on 16 held-out skies.
Every problem reaches F*(1 + 1e-6) from both starts, the network's start is
taken (its objective is below the zero image's), and the mean iteration
count does not grow.  Measured on 256 held-out skies: 1959 -> 1947 mean
iterations, 87.5 % of problems need fewer; the gain is small because the
slowest directions are the poorly sampled uv ones, which a prediction from
the dirty image and beam does not pin down either."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_config4_warm_start_on_held_out_skies(gpulib):
    from sparseimaging_b200 import warmstart
    net = warmstart.load(256)
    ev = warmstart.evaluate(net, list(range(90000, 90016)), nx=256, batch=16, fstar_iters=4000)
    net.close()
    s = ev["summary"]
    assert s["reached_zero"] == s["reached_warm"] == 16
    assert s["used_start"] >= 12
    assert s["mean_iters_warm"] <= s["mean_iters_zero"]
