"""Movie solved as one problem (mfista_nufft_movie): frames coupled by the
temporal term lambda_t sum_b |x_b - x_{b+1}|^2 / dt_b with one joint step
size, backtracking test and stopping rule (matlab/MFISTA_movie_eht.m).

Checked against oracle/movie_oracle.py (FP64, other summation orders: 1e-8
on the images after 200 iterations), against the batched solver for one
frame without the temporal term (the same bits: the joint control adds the
same sums in the same order), and for the frame times: doubling every time
step equals halving lambda_t (exact scalings by 2)."""
import numpy as np
import pytest

from conftest import rel
from oracle import movie_oracle as MO

pytestmark = pytest.mark.gpu


def _movie(T, nx=32, seed=4):
    from sparseimaging_b200 import synth
    fr = synth.movie_problem(n_frames=T, nx=nx, seed=seed, m_range=(150, 300))
    cat = lambda a: np.concatenate([getattr(f, a) for f in fr])
    off = np.concatenate([[0], np.cumsum([f.m for f in fr])]).astype(np.int32)
    geo = (cat("u_dx"), cat("v_dy"), cat("vis_r"), cat("vis_i"), cat("vis_std"))
    return fr, geo, off


def _params(gpulib, fr, nx):
    f = fr[0]
    w2 = 1 / f.vis_std ** 2
    g0 = gpulib.nufft_adjoint(f.u_dx, f.v_dy, nx, nx, f.vis_r * w2, f.vis_i * w2)
    lam = 1e-2 * float(np.abs(g0).max())
    lip = max(gpulib.nufft_lipschitz(g.u_dx, g.v_dy, g.vis_std, nx, nx, iters=20) for g in fr)
    return lam, lip


def test_movie_matches_oracle(gpulib):
    nx, T = 32, 4
    fr, geo, off = _movie(T, nx)
    lam, lip = _params(gpulib, fr, nx)
    lt = 5.0 * lam
    X, R, tcost = gpulib.nufft_movie(*geo, off, nx, nx, lam, 1e-2 * lam, lt, lip, 200, 0.0)
    frames = [(f.u_dx, f.v_dy, f.vis_r, f.vis_i, f.vis_std) for f in fr]
    Xo, it, c, cost = MO.movie(frames, nx, nx, lam, 1e-2 * lam, lt, lip, 200, 0.0)
    assert all(r["ITER"] == it for r in R)
    assert rel(X, Xo) < 1e-8
    assert abs(tcost - lt * MO.d_x(Xo, np.ones(T - 1))) <= 1e-8 * tcost
    total = sum(r["finalcost"] for r in R) + tcost
    assert abs(total - cost[-1]) <= 1e-8 * cost[-1] or total <= cost[-1]


def test_single_frame_equals_batch_solve(gpulib):
    nx = 32
    fr, geo, off = _movie(1, nx, seed=6)
    lam, lip = _params(gpulib, fr, nx)
    eps = 1e-6
    f = fr[0]
    scaled = (f.vis_r @ f.vis_r + f.vis_i @ f.vis_i) * eps / f.m
    prob = [dict(lambda_l1=lam, lambda_tsv=1e-2 * lam, cinit=lip, maxiter=300, nonneg_flag=1)]
    Xb, Rb = gpulib.nufft_batch(*geo, nx, nx, prob, eps, pt_off=off)
    Xm, Rm, tc = gpulib.nufft_movie(*geo, off, nx, nx, lam, 1e-2 * lam, 0.0, lip, 300, scaled)
    assert Rm[0]["ITER"] == Rb[0]["ITER"]
    assert np.array_equal(Xm[0], Xb[0])
    assert tc == 0.0


def test_frame_times_scale_the_temporal_weight(gpulib):
    nx, T = 32, 3
    fr, geo, off = _movie(T, nx, seed=8)
    lam, lip = _params(gpulib, fr, nx)
    a = gpulib.nufft_movie(*geo, off, nx, nx, lam, 1e-2 * lam, 4.0 * lam, lip, 120, 0.0,
                           t_list=2.0 * np.arange(1, T + 1))
    b = gpulib.nufft_movie(*geo, off, nx, nx, lam, 1e-2 * lam, 2.0 * lam, lip, 120, 0.0)
    assert np.array_equal(a[0], b[0])
    assert [r["ITER"] for r in a[1]] == [r["ITER"] for r in b[1]]


def test_movie_c_box_matches_oracle(gpulib):
    """c_box as the matlab code applies it: xinit .* c_box, and every
    thresholded image times c_box (a support mask with fractional edges)."""
    nx, T = 32, 3
    fr, geo, off = _movie(T, nx, seed=11)
    lam, lip = _params(gpulib, fr, nx)
    lt = 5.0 * lam
    yy, xx = np.divmod(np.arange(nx * nx), nx)
    r2 = (yy - nx / 2) ** 2 + (xx - nx / 2) ** 2
    box = np.where(r2 <= (nx / 3) ** 2, 1.0, np.where(r2 <= (nx / 2.5) ** 2, 0.5, 0.0))
    x0 = np.full(nx * nx, 1e-4)
    X, R, tcost = gpulib.nufft_movie(*geo, off, nx, nx, lam, 1e-2 * lam, lt, lip, 200, 0.0, xinit=x0, c_box=box)
    frames = [(f.u_dx, f.v_dy, f.vis_r, f.vis_i, f.vis_std) for f in fr]
    Xo, it, c, cost = MO.movie(frames, nx, nx, lam, 1e-2 * lam, lt, lip, 200, 0.0, xinit=x0, c_box=box)
    assert all(r["ITER"] == it for r in R)
    assert rel(X, Xo) < 1e-8
    assert np.all(X[:, box == 0] == 0)


def test_movie_fp32_form(gpulib):
    """The FP32 form of the joint movie (corrected FP32 NUFFTs, FP64 control)
    reaches the FP64 form's objective: the same stopping rule on the summed
    objective, final objectives within 1e-6 relative."""
    nx, T = 32, 4
    fr, geo, off = _movie(T, nx, seed=13)
    lam, lip = _params(gpulib, fr, nx)
    lt = 5.0 * lam
    out = {}
    for prec in (gpulib.FP64, gpulib.FP32):
        X, R, tcost = gpulib.nufft_movie(*geo, off, nx, nx, lam, 1e-2 * lam, lt, lip, 3000, 1e-9, precision=prec)
        out[prec] = (X, sum(r["finalcost"] for r in R) + tcost, R[0]["ITER"])
    f64, f32 = out[gpulib.FP64][1], out[gpulib.FP32][1]
    assert abs(f32 - f64) <= 1e-6 * f64
    assert rel(out[gpulib.FP32][0], out[gpulib.FP64][0]) < 1e-2


def test_movie_rejects_bad_frame_times(gpulib):
    nx, T = 32, 3
    fr, geo, off = _movie(T, nx, seed=8)
    with pytest.raises(gpulib.MfistaError):
        gpulib.nufft_movie(*geo, off, nx, nx, 1.0, 0.0, 1.0, 1.0, 10, 0.0, t_list=[1.0, 1.0, 2.0])
