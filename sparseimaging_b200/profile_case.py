"""Short, bounded runs of the solver for profiling (ncu) and timing.

    python -m sparseimaging_b200.profile_case --case lambda-grid --precision 64 --iters 20
    python -m sparseimaging_b200.profile_case --case lambda-grid --kernel 1 --reps 3

For ncu, pass --gmax/--lip (bench.py's values for the lambda grid are
gmax 4011856.19 and lip 2.156e10) so that no setup kernels run before the
plan's, and set MFISTA_HOST_LOOP=1: ncu profiles the kernels of an ordinary
graph but not those inside a conditional WHILE body.

--case lambda-grid: the 128x128, M = 8100, 64-problem lambda grid that
bench.py times; --case config0: the 64x64 single problem; --case dft: the
batched DFT GEMMs (A 8000 x 4096, --problems right-hand sides) timed alone,
--precision 64 for FP64 or 32 for the tensor-core split-BF16 form.  Without
--kernel it runs one batched solve of --iters MFISTA iterations; with
--kernel k it times that operator kernel alone (see mfista_plan_profile).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="lambda-grid", choices=["lambda-grid", "config0", "dft"])
    ap.add_argument("--precision", type=int, default=64, choices=[32, 64])
    ap.add_argument("--iters", type=int, default=20)
    ap.add_argument("--kernel", type=int, default=-1)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--problems", type=int, default=64)
    ap.add_argument("--gmax", type=float, default=0.0,
                    help="max|A^H W^2 y| (skips its GPU computation when given)")
    ap.add_argument("--lip", type=float, default=0.0,
                    help="Lipschitz estimate for cinit (skips the power iteration when given)")
    ap.add_argument("--shapes", default="",
                    help="launch shapes interp_ppw,spread_cluster,rows_per_cta,cols_per_cta (0 keeps a default)")
    a = ap.parse_args()
    os.environ.setdefault("MFISTA_QUIET", "1")
    import sparseimaging_b200 as si
    from sparseimaging_b200 import synth
    if a.case == "dft":
        # 64x64 image, 4000 visibilities from 10 stations: A is 8000 x 4096
        p = synth.dft_problem()
        prec = {64: si.FP64, 32: si.BF16X3}[a.precision]
        out = {"case": "dft", "precision": "fp64" if prec == si.FP64 else "bf16x3", "M": p.A.shape[0],
               "N": p.A.shape[1], "problems": a.problems}
        for k in (0, 1) if a.kernel < 0 else (a.kernel,):
            ms, by = si.dft_profile(p.A, a.problems, k, precision=prec, reps=a.reps)
            out[f"kernel{k}"] = {"ms_per_launch": ms, "bytes_per_launch": by, "gbs": by / ms / 1e6,
                                 "tflops": 2.0 * p.A.shape[0] * p.A.shape[1] * a.problems / ms / 1e9}
        print(json.dumps(out))
        return
    p = synth.lambda_grid_problem() if a.case == "lambda-grid" else synth.config0()
    nx = p.nx
    w2 = 1 / p.vis_std ** 2
    gmax, lip = a.gmax, a.lip
    if gmax <= 0:
        g0 = si.nufft_adjoint(p.u_dx, p.v_dy, nx, nx, p.vis_r * w2, p.vis_i * w2)
        gmax = float(np.abs(g0).max())
    if lip <= 0:
        lip = si.nufft_lipschitz(p.u_dx, p.v_dy, p.vis_std, nx, nx, iters=10)
    grid = synth.lambda_grid(gmax, 8, 8, 1e-4, 1.0)[: a.problems]
    probs = [dict(lambda_l1=float(l1), lambda_tsv=float(lt), cinit=lip, maxiter=a.iters, nonneg_flag=1)
             for l1, lt in grid]
    plan = si.Plan(p.u_dx, p.v_dy, p.vis_r, p.vis_i, p.vis_std, nx, nx, len(probs), precision=a.precision)
    if a.shapes:
        vals = [int(v) for v in a.shapes.split(",")]
        plan.set_shapes(**dict(zip(si.Plan.SHAPE_KEYS, vals)))
    plan.set_problems(probs, 0.0)
    out = {"case": a.case, "precision": a.precision, "problems": len(probs), "M": p.m, "shapes": plan.shapes()}
    if a.kernel >= 0:
        ms, by = plan.profile(a.kernel, a.reps)
        out.update(kernel=a.kernel, ms_per_launch=ms, bytes_per_launch=by, gbs=by / ms / 1e6)
    else:
        t = time.perf_counter()
        plan.run()
        _, R = plan.fetch(want_x=False)
        out.update(iters=a.iters, seconds=time.perf_counter() - t, kernel_launches=plan.kernel_launches,
                   device_loop=plan.device_loop)
    plan.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
