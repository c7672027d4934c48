"""F* (converged FP64 objective) of the 64-problem DFT lambda grid.

Run once on a GPU (`python tests/golden/make_dft_fstar.py`): the library's
FP64 batched DFT solver runs the 64 problems (64x64 image, 4000 visibilities
from 10 stations, stacked real/imaginary A of 8000 x 4096, lambda_l1 and
lambda_tsv on an 8x8 log grid over 1e-4 .. 1 of max|A^T y|, nonnegative)
for FSTAR_ITERS iterations with the stop rule off (eps = 0); the objectives,
the workload parameters and the FP64 iterations to F*(1 + 1e-6) are written
to tests/golden/dft_lambda_grid_fstar.json, which bench.py checks before use.
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


def dft_workload():
    from sparseimaging_b200 import synth
    p = synth.dft_problem()
    A, y = p.A, p.y
    gmax = float(np.abs(A.T @ y).max())
    v = np.random.default_rng(0).standard_normal(A.shape[1])
    for _ in range(50):  # power iteration for ||A||^2 (cinit)
        v = A.T @ (A @ v)
        v /= np.linalg.norm(v)
    lip = float(np.linalg.norm(A @ v) ** 2)
    grid = synth.lambda_grid(gmax, 8, 8, 1e-4, 1.0)
    return p, gmax, lip, grid


def problems(grid, lip, maxiter, targets=None):
    return [dict(lambda_l1=float(l1), lambda_tsv=float(lt), cinit=lip, maxiter=maxiter, nonneg_flag=1,
                 target_cost=0.0 if targets is None else float(targets[b])) for b, (l1, lt) in enumerate(grid)]


def main():
    os.environ.setdefault("MFISTA_QUIET", "1")
    import sparseimaging_b200 as si
    p, gmax, lip, grid = dft_workload()
    t = time.time()
    _, R = si.dft_batch(p.y, p.A, p.nx, p.nx, problems(grid, lip, FSTAR_ITERS), 0.0)
    secs = time.time() - t
    fstar = [r["finalcost"] for r in R]
    targets = [f * (1 + 1e-6) for f in fstar]
    _, R2 = si.dft_batch(p.y, p.A, p.nx, p.nx, problems(grid, lip, FSTAR_ITERS, targets), 0.0)
    out = {"nx": p.nx, "M": int(p.A.shape[0]), "N": int(p.A.shape[1]), "gmax": gmax, "lip": lip,
           "iters": FSTAR_ITERS, "seconds": secs, "fstar": fstar, "iters_run": [r["ITER"] for r in R],
           "iters_to_target_fp64": [r["ITER"] for r in R2]}
    json.dump(out, open(os.path.join(HERE, "dft_lambda_grid_fstar.json"), "w"), indent=1)
    print(json.dumps({k: v for k, v in out.items() if not isinstance(v, list)}))


if __name__ == "__main__":
    main()
