"""Checks F* of the lambda-grid fixture against the reference itself.

F* in tests/golden/lambda_grid_fstar.json comes from this library's FP64
batched solver run for 20000 iterations.  Here the reference C, compiled
unchanged (oracle/_ref, FFTW/BLAS shims), runs the same 20000 iterations
(stopping rule off: eps = 0) on four problems of the grid on the host
cores, and the relative differences of its final objective from F* are
written into the fixture (`fstar_reference_check`).  Run where the
reference has been built (about 15 minutes on 4 cores):

    python tests/golden/check_fstar_reference.py
"""
from __future__ import annotations

import json
import multiprocessing as mp
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

PICKS = [0, 9, 27, 45]


def _solve(args):
    b, iters = args
    sys.path.insert(0, ROOT)
    sys.path.insert(0, HERE)
    import bench
    from make_golden import quiet_call
    from oracle import ref_ctypes as R
    fx = json.load(open(os.path.join(HERE, "lambda_grid_fstar.json")))
    p = bench.workload(seed=fx["seed"])
    lam1, lamt = bench.lam_grid(fx["gmax"])[b]
    _, res = quiet_call(R.core_nufft, p.u_dx, p.v_dy, p.vis_r, p.vis_i, p.vis_std, p.nx, p.nx, iters, 0.0,
                        float(lam1), 0.0, float(lamt), fx["lip"], nonneg_flag=1)
    return b, res.finalcost, res.ITER


def main():
    path = os.path.join(HERE, "lambda_grid_fstar.json")
    fx = json.load(open(path))
    ctx = mp.get_context("spawn")
    with ctx.Pool(len(PICKS)) as pool:
        out = pool.map(_solve, [(b, fx["iters"]) for b in PICKS])
    rows = []
    for b, cost, it in out:
        f = fx["fstar"][b]
        rows.append({"problem": b, "reference_cost": cost, "reference_iters": it, "fstar": f,
                     "rel_diff": (cost - f) / f})
    fx["fstar_reference_check"] = rows
    json.dump(fx, open(path, "w"), indent=1)
    print(json.dumps(rows, indent=1))


if __name__ == "__main__":
    main()
