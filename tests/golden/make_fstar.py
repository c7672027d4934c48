"""F* and x* (converged FP64 objective and image) of every problem of
bench.py's lambda grid.

Run once on a GPU (`python tests/golden/make_fstar.py`): the library's FP64
batched solver runs the 64 problems for FSTAR_ITERS iterations with the
reference stop rule disabled (eps = 0); the final objectives are written to
tests/golden/lambda_grid_fstar.json together with the workload parameters
they belong to, which bench.py checks before using them, and the final
images x* (float32) to tests/golden/lambda_grid_xstar.npz.  A second run of
LONG_ITERS iterations measures how far F* and x* still are from the
optimum: its objective and image differences are stored beside them
(`fstar_long_rel`, `xstar_long_rel`), so that an image error measured
against x* can be read against the uncertainty of x* itself.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

FSTAR_ITERS = 20000
LONG_ITERS = 60000


def _solve(si, bench, p, grid, lip, iters, targets=None):
    nx = p.nx
    plan = si.Plan(p.u_dx, p.v_dy, p.vis_r, p.vis_i, p.vis_std, nx, nx, len(grid), precision=si.FP64)
    plan.set_problems(bench.problems(grid, lip, iters, targets), 0.0)
    plan.run()
    X, R = plan.fetch(want_x=True)
    plan.close()
    return X, R


def main():
    os.environ.setdefault("MFISTA_QUIET", "1")
    import bench
    import sparseimaging_b200 as si
    p = bench.workload(seed=7)
    nx = p.nx
    w2 = 1 / p.vis_std ** 2
    g0 = si.nufft_adjoint(p.u_dx, p.v_dy, nx, nx, p.vis_r * w2, p.vis_i * w2)
    gmax = float(np.abs(g0).max())
    lip = si.nufft_lipschitz(p.u_dx, p.v_dy, p.vis_std, nx, nx, iters=20)
    grid = bench.lam_grid(gmax)
    t = time.time()
    X, R = _solve(si, bench, p, grid, lip, FSTAR_ITERS)
    secs = time.time() - t
    fstar = [r["finalcost"] for r in R]
    # iterations the FP64 solver needs to come within 1e-6 of F* (these are
    # the iterations the reference C needs too: same FP64 trajectory)
    targets = [f * (1 + bench.REL_OBJ) for f in fstar]
    _, R2 = _solve(si, bench, p, grid, lip, FSTAR_ITERS, targets)
    XL, RL = _solve(si, bench, p, grid, lip, LONG_ITERS)
    f_rel = [(a["finalcost"] - b["finalcost"]) / b["finalcost"] for a, b in zip(R, RL)]
    x_rel = [float(np.linalg.norm(X[b] - XL[b]) / max(np.linalg.norm(XL[b]), 1e-300)) for b in range(len(grid))]
    np.savez_compressed(os.path.join(HERE, "lambda_grid_xstar.npz"), xstar=X.astype(np.float32),
                        iters=np.int32(FSTAR_ITERS))
    out = {"seed": 7, "nx": nx, "M": p.m, "gmax": gmax, "lip": lip, "iters": FSTAR_ITERS,
           "seconds": secs, "long_iters": LONG_ITERS, "xstar_file": "lambda_grid_xstar.npz",
           "fstar": fstar, "iters_run": [r["ITER"] for r in R],
           "iters_to_target_fp64": [r["ITER"] for r in R2],
           "fstar_long_rel": f_rel, "xstar_long_rel": x_rel}
    json.dump(out, open(os.path.join(HERE, "lambda_grid_fstar.json"), "w"), indent=1)
    summ = {k: v for k, v in out.items() if not isinstance(v, list)}
    summ.update(max_fstar_long_rel=max(f_rel), max_xstar_long_rel=max(x_rel),
                median_xstar_long_rel=float(np.median(x_rel)))
    print(json.dumps(summ))


if __name__ == "__main__":
    main()
