"""The movie oracle (oracle/movie_oracle.py, a restatement of the
reference's matlab/MFISTA_movie_eht.m, which cannot run here) pinned where
it must coincide with the C reference's MFISTA loop: one frame, no temporal
term, the scaled eps of mfista_imaging_core_nufft.  Plus properties of the
coupled case: a monotone objective, and a temporal term that shrinks as
lambda_t grows."""
import numpy as np

from oracle import mfista_oracle as R
from oracle import movie_oracle as MO
from sparseimaging_b200 import synth


def _frames(T, nx=16, seed=2):
    fr = synth.movie_problem(n_frames=T, nx=nx, seed=seed, m_range=(60, 120))
    return fr, [(f.u_dx, f.v_dy, f.vis_r, f.vis_i, f.vis_std) for f in fr]


def _lams(f, nx):
    plan = R.NufftPlan(f.u_dx, f.v_dy, nx, nx)
    w2 = 1 / f.vis_std ** 2
    g0 = plan.adjoint(f.vis_r * w2, f.vis_i * w2)
    lam = 1e-2 * float(np.abs(g0).max())
    lip = R.lipschitz_nufft(plan, 1 / f.vis_std, iters=20)
    return lam, lip


def test_single_frame_equals_reference_loop():
    nx = 16
    fr, frames = _frames(1, nx)
    f = fr[0]
    lam, lip = _lams(f, nx)
    eps = 1e-7
    x_ref, res = R.imaging_core_nufft(f.u_dx, f.v_dy, f.vis_r, f.vis_i, f.vis_std, nx, nx, 300, eps, lam, 0.0,
                                      1e-2 * lam, lip, np.zeros(nx * nx), 1)
    scaled = (f.vis_r @ f.vis_r + f.vis_i @ f.vis_i) * eps / f.vis_r.size
    X, it, c, _ = MO.movie(frames, nx, nx, lam, 1e-2 * lam, 0.0, lip, 300, scaled)
    assert it == res["ITER"]
    assert np.array_equal(X[0], x_ref)


def test_coupled_movie_properties():
    nx = 16
    fr, frames = _frames(3, nx)
    lam, lip = _lams(fr[0], nx)
    lip *= 1.5
    out = {}
    for lt in (0.0, 10.0 * lam):
        X, it, c, cost = MO.movie(frames, nx, nx, lam, 1e-2 * lam, lt, lip, 150, 0.0)
        assert np.all(np.diff(cost) <= 0)          # MFISTA keeps the objective monotone
        out[lt] = MO.d_x(X, np.ones(2))
    assert out[10.0 * lam] < out[0.0]


def test_c_box_support_and_scaling():
    """c_box (matlab/MFISTA_movie_eht.m:46, :143-146): ones change nothing,
    a 0/1 mask keeps the pixels outside it at zero, and the frames stay
    monotone with fractional weights."""
    nx = 16
    fr, frames = _frames(2, nx, seed=5)
    lam, lip = _lams(fr[0], nx)
    lip *= 1.5
    args = (frames, nx, nx, lam, 1e-2 * lam, 5.0 * lam, lip, 80, 0.0)
    X0, it0, _, _ = MO.movie(*args)
    X1, it1, _, _ = MO.movie(*args, c_box=np.ones(nx * nx))
    assert it0 == it1 and np.array_equal(X0, X1)
    yy, xx = np.divmod(np.arange(nx * nx), nx)
    mask = ((yy - nx / 2) ** 2 + (xx - nx / 2) ** 2 <= (nx / 3) ** 2).astype(np.float64)
    Xm, _, _, cost = MO.movie(*args, c_box=mask, xinit=np.full(nx * nx, 1e-3))
    assert np.all(Xm[:, mask == 0] == 0)
    assert np.any(Xm[:, mask == 1] != 0)
    assert np.all(np.diff(cost) <= 0)
    w = 0.5 + 0.5 * mask
    Xw, _, _, cost = MO.movie(*args, c_box=w)
    assert np.all(np.diff(cost) <= 0)
