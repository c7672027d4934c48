"""Image error of the batched FP32 form against the converged FP64 images.

The 64-problem lambda grid that bench.py times (128 x 128, M = 8100) is
solved to F*(1 + 1e-6) by the batched FP64 form and by the chosen FP32 form
(FP32 NUFFT/FFT with FP64 anchor correction).  tests/golden/make_fstar.py
stored F* and the converged images x* (FP64, 20000 iterations).

At that objective tolerance the solution is not determined to 1e-4 in
image space: the FP64 solver's own images lie 3e-3 to 2e-1 (relative L2)
from x* on this grid, because the poorly sampled uv directions barely move
the objective.  What the precision form must not do is add error of its
own, so the test holds the FP32 form's distance to x* to that of the FP64
form, problem by problem: err32 <= max(1e-4, 1.05 err64).
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu


def _errors(X, xs):
    out = []
    for b in range(len(xs)):
        n = np.linalg.norm(xs[b])
        out.append(float(np.linalg.norm(X[b] - xs[b]) / n) if n > 0 else float(np.abs(X[b]).max()))
    return np.array(out)


def test_fp32_form_image_error_matches_fp64(gpulib):
    import sys
    sys.path.insert(0, ROOT)
    import bench
    fx = json.load(open(os.path.join(GOLDEN, "lambda_grid_fstar.json")))
    xs = np.load(os.path.join(GOLDEN, fx["xstar_file"]))["xstar"].astype(np.float64)
    p = bench.workload(seed=fx["seed"])
    assert p.m == fx["M"] and p.nx == fx["nx"]
    fstar = np.array(fx["fstar"])
    targets = fstar * (1 + bench.REL_OBJ)
    grid = bench.lam_grid(fx["gmax"])
    probs = bench.problems(grid, fx["lip"], bench.MAXITER_CAP, targets)
    geo = (p.u_dx, p.v_dy, p.vis_r, p.vis_i, p.vis_std, p.nx, p.nx)
    X64, R64 = gpulib.nufft_batch(*geo, probs, 0.0, precision=gpulib.FP64)
    X32, R32 = gpulib.nufft_batch(*geo, probs, 0.0, precision=gpulib.FP32)
    for R in (R64, R32):
        assert all(r["finalcost"] <= t for r, t in zip(R, targets))
    e64, e32 = _errors(X64, xs), _errors(X32, xs)
    nz = np.array([np.linalg.norm(x) > 0 for x in xs])
    # the zero solutions: the grid's largest lambda_l1 is max|A^H y| itself,
    # where FP64 keeps x = 0 exactly and an FP32 gradient may pass the
    # threshold by a rounding (measured: one pixel at 7.8e-12, 1e-8 of the
    # images' peak); hold it to 1e-6 of the median peak of x*
    scale = float(np.median([np.abs(x).max() for x in xs[nz]]))
    assert np.all(e64[~nz] == 0) and np.all(e32[~nz] <= 1e-6 * scale)
    bound = np.maximum(1e-4, 1.05 * e64)
    bad = [(b, e32[b], e64[b]) for b in range(len(xs)) if e32[b] > bound[b]]
    assert not bad, bad
