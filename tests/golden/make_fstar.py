"""F* (converged FP64 objective) of every problem of bench.py's lambda grid.

Run once on a GPU (`python tests/golden/make_fstar.py`): the library's FP64
batched solver runs the 64 problems for FSTAR_ITERS iterations with the
reference stop rule disabled (eps = 0); the final objectives are written to
tests/golden/lambda_grid_fstar.json together with the workload parameters
they belong to, which bench.py checks before using them.
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
    plan = si.Plan(p.u_dx, p.v_dy, p.vis_r, p.vis_i, p.vis_std, nx, nx, len(grid), precision=si.FP64)
    plan.set_problems(bench.problems(grid, lip, FSTAR_ITERS), 0.0)
    plan.run()
    _, R = plan.fetch(want_x=False)
    secs = time.time() - t
    fstar = [r["finalcost"] for r in R]
    # iterations the FP64 solver needs to come within 1e-6 of F* (these are
    # the iterations the reference C needs too: same FP64 trajectory)
    targets = [f * (1 + bench.REL_OBJ) for f in fstar]
    plan.set_problems(bench.problems(grid, lip, FSTAR_ITERS, targets), 0.0)
    plan.run()
    _, R2 = plan.fetch(want_x=False)
    plan.close()
    out = {"seed": 7, "nx": nx, "M": p.m, "gmax": gmax, "lip": lip, "iters": FSTAR_ITERS,
           "seconds": secs, "fstar": fstar, "iters_run": [r["ITER"] for r in R],
           "iters_to_target_fp64": [r["ITER"] for r in R2]}
    json.dump(out, open(os.path.join(HERE, "lambda_grid_fstar.json"), "w"), indent=1)
    print(json.dumps({k: v for k, v in out.items() if not isinstance(v, list)}))


if __name__ == "__main__":
    main()
