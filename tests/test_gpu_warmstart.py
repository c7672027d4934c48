"""What the trained warm start gains on the benchmark's lambda grid.

The committed network (sparseimaging_b200/data/unet_warmstart_128.npy,
trained on the GPU by `python -m sparseimaging_b200.warmstart --train` from
FP64 solutions of 384 seeded skies other than the benchmark's) predicts an
initial image from the dirty image and dirty beam; each problem starts from
it only when its objective there is below the zero image's.  The batched
FP32 solver (FP64 anchor correction) then runs every problem to its target
F*(1 + 1e-6) from the F* fixture.  Measured gain on this grid is small: the
mean iteration count drops by about 2 % and the slowest problem (which sets
the batch time) is unchanged; the test pins that it is not negative."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_warm_start_reaches_every_target_with_fewer_iterations(gpulib):
    import sys
    sys.path.insert(0, ROOT)
    import bench
    from sparseimaging_b200 import warmstart as ws
    p = bench.workload(seed=7)
    nx = p.nx
    w2 = 1 / p.vis_std ** 2
    g0 = gpulib.nufft_adjoint(p.u_dx, p.v_dy, nx, nx, p.vis_r * w2, p.vis_i * w2)
    lip = gpulib.nufft_lipschitz(p.u_dx, p.v_dy, p.vis_std, nx, nx, iters=20)
    grid = bench.lam_grid(float(np.abs(g0).max()))
    fx = json.load(open(bench.FSTAR_FILE))
    targets = np.array(fx["fstar"]) * (1 + bench.REL_OBJ)
    geo = (p.u_dx, p.v_dy, p.vis_r, p.vis_i, p.vis_std, nx, nx)
    probs = bench.problems(grid, lip, bench.MAXITER_CAP, targets)
    net = ws.load(nx)
    xw = ws.predict(net, *geo[:5], nx)
    net.close()
    assert np.all(xw >= 0) and np.isfinite(xw).all()
    x0, used = ws.choose_starts(geo, probs, xw)
    assert used.sum() >= 16            # the start beats zero for most small-lambda problems
    _, Rz = gpulib.nufft_batch(*geo, probs, 0.0, precision=gpulib.FP32)
    _, Rw = gpulib.nufft_batch(*geo, probs, 0.0, xinit=x0, precision=gpulib.FP32)
    for r, t in zip(Rw, targets):
        assert r["finalcost"] <= t     # MFISTA still judges: every problem reaches its target
    it_z = np.array([r["ITER"] for r in Rz])
    it_w = np.array([r["ITER"] for r in Rw])
    print(f"warm start on {int(used.sum())}/64 problems: mean iterations {it_z.mean():.1f} -> {it_w.mean():.1f}, "
          f"max {it_z.max()} -> {it_w.max()}")
    assert it_w.mean() < it_z.mean()
    assert np.all(it_w[~used] == it_z[~used])  # zero-start problems are untouched
