"""A movie of 48 frames with uneven visibility counts in one batched solve.

Frames of a rotating-spot ring (128x128, 6-10 stations, M from ~1400 to
~11700 per frame, 2 % noise) are independent L1+TSV problems solved in ONE
launch of the batched solver (per-problem point ranges, per-problem
backtracking state and convergence masks).  The FP32 form (FP64 anchor
correction) must bring every frame to the FP64 batch's objective (after
1500 FP64 iterations) within 1e-6, and each FP64 frame must match its own
single-problem solve to rounding (the kernels never mix frames; the
per-frame-range kernels sum in another order than the single problem's
shared-geometry kernels, which moves 200-iteration images by ~3e-10).  Images that agree to
1e-6 in objective still differ by a few percent here (measured: median
4e-2, max 6e-2 relative L2): after 1500 iterations the FP64 run sits on a
flat part of the objective, and the FP32 run stops at the first point of
that valley that reaches the target."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


def _movie(gpulib):
    from sparseimaging_b200 import synth
    frames = synth.movie_problem()
    nx = frames[0].nx
    probs = []
    for f in frames:
        w2 = 1 / f.vis_std ** 2
        g0 = gpulib.nufft_adjoint(f.u_dx, f.v_dy, nx, nx, f.vis_r * w2, f.vis_i * w2)
        lam = 1e-2 * float(np.abs(g0).max())
        lip = gpulib.nufft_lipschitz(f.u_dx, f.v_dy, f.vis_std, nx, nx, iters=10)
        probs.append(dict(lambda_l1=lam, lambda_tsv=1e-3 * lam, cinit=lip, maxiter=1500, nonneg_flag=1))
    cat = lambda a: np.concatenate([getattr(f, a) for f in frames])
    off = np.concatenate([[0], np.cumsum([f.m for f in frames])]).astype(np.int32)
    geo = (cat("u_dx"), cat("v_dy"), cat("vis_r"), cat("vis_i"), cat("vis_std"), nx, nx)
    return frames, probs, geo, off


def test_movie_batch_fp32_reaches_fp64_objective_per_frame(gpulib):
    frames, probs, geo, off = _movie(gpulib)
    X64, R64 = gpulib.nufft_batch(*geo, probs, 0.0, pt_off=off)
    assert [r["M"] for r in R64] == [f.m // 2 for f in frames]  # RESULT.M = M / 2 as in the reference
    targets = [r["finalcost"] * (1 + 1e-6) for r in R64]
    probs32 = [dict(p, maxiter=6000, target_cost=t) for p, t in zip(probs, targets)]
    X32, R32 = gpulib.nufft_batch(*geo, probs32, 0.0, pt_off=off, precision=gpulib.FP32)
    errs = []
    for b, (r, t) in enumerate(zip(R32, targets)):
        assert r["finalcost"] <= t, (b, r["finalcost"], t)
        errs.append(rel(X32[b], X64[b]))
    print(f"movie: 48 frames, per-frame image error of the FP32 form vs FP64: median {np.median(errs):.2e}, "
          f"max {max(errs):.2e}")
    assert max(errs) < 1e-1


def test_movie_batch_fp64_frames_equal_single_solves(gpulib):
    frames, probs, geo, off = _movie(gpulib)
    pick = [0, 17, 47]
    sub = [frames[i] for i in pick]
    cat = lambda a: np.concatenate([getattr(f, a) for f in sub])
    offs = np.concatenate([[0], np.cumsum([f.m for f in sub])]).astype(np.int32)
    nx = frames[0].nx
    sp = [dict(probs[i], maxiter=200) for i in pick]
    X, R = gpulib.nufft_batch(cat("u_dx"), cat("v_dy"), cat("vis_r"), cat("vis_i"), cat("vis_std"), nx, nx, sp,
                              1e-5, pt_off=offs)
    for k, i in enumerate(pick):
        f = frames[i]
        x, r = gpulib.imaging_core_nufft(f.u_dx, f.v_dy, f.vis_r, f.vis_i, f.vis_std, nx, nx, 200, 1e-5,
                                         sp[k]["lambda_l1"], 0.0, sp[k]["lambda_tsv"], sp[k]["cinit"])
        assert R[k]["ITER"] == r["ITER"]
        assert rel(X[k], x) < 1e-8
        assert abs(R[k]["finalcost"] - r["finalcost"]) <= 1e-12 * r["finalcost"]
