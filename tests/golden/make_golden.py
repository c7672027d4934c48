"""Generates the golden fixtures in tests/golden/ from the reference itself.

Run here (where the reference sources exist) after `make -C oracle`:

    python tests/golden/make_golden.py

Every fixture stores its exact inputs and the outputs of the reference C
solvers compiled unchanged (oracle/_ref/libmfista_ref.so, FFTW/BLAS shims),
so the GPU tests can compare against the reference without the reference
being present.  cinit comes from the oracle's power iteration.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from oracle import mfista_oracle as O  # noqa: E402
from oracle import ref_ctypes as R     # noqa: E402
from sparseimaging_b200 import synth   # noqa: E402

RES_KEYS = ["M", "N", "NX", "NY", "N_active", "maxiter", "ITER", "nonneg", "lambda_l1",
            "lambda_tv", "lambda_tsv", "sq_error", "mean_sq_error", "l1cost", "tvcost",
            "tsvcost", "finalcost", "Lip_const"]


def res_arr(res):
    d = res.as_dict()
    return np.array([float(d[k]) for k in RES_KEYS])


def quiet_call(fn, *a, **k):
    """The reference prints every 10 iterations; silence fd 1 during calls."""
    sys.stdout.flush()
    fd = os.dup(1)
    dn = os.open(os.devnull, os.O_WRONLY)
    os.dup2(dn, 1)
    try:
        return fn(*a, **k)
    finally:
        os.dup2(fd, 1)
        os.close(fd)
        os.close(dn)


def make_c0():
    p = synth.config0()
    plan = O.NufftPlan(p.u_dx, p.v_dy, 64, 64)
    w = 1 / p.vis_std
    g0 = plan.adjoint(p.vis_r * w * w, p.vis_i * w * w)
    lam1 = 1e-2 * np.abs(g0).max()
    lamt = 1e-3 * lam1
    cinit = O.lipschitz_nufft(plan, w)
    out = dict(u=p.u_dx, v=p.v_dy, vis_r=p.vis_r, vis_i=p.vis_i, vis_std=p.vis_std, sky=p.sky.ravel(),
               lam1=lam1, lamt=lamt, cinit=cinit)
    # operators
    ref = R.RefNufft(p.u_dx, p.v_dy, 64, 64)
    fr, fi = ref.forward(p.sky.ravel())
    rng = np.random.default_rng(11)
    rr, ri = rng.standard_normal(p.m), rng.standard_normal(p.m)
    out.update(fwd_r=fr, fwd_i=fi, adj_in_r=rr, adj_in_i=ri, adj_out=ref.adjoint(rr, ri))
    ref.close()
    args = (p.u_dx, p.v_dy, p.vis_r, p.vis_i, p.vis_std, 64, 64)
    for mi in (400, 1000):
        x, res = quiet_call(R.core_nufft, *args, mi, 1e-5, lam1, 0.0, lamt, cinit, nonneg_flag=1)
        out[f"x_{mi}"] = x
        out[f"res_{mi}"] = res_arr(res)
    # the reference's own spread under 1-ulp-level input perturbations
    dx, dc = 0.0, 0.0
    for k, s in enumerate((1 + 1e-15, 1 - 1e-15, 1 + 3e-15)):
        vr = p.vis_r.copy()
        vr[k] *= s
        x2, r2 = quiet_call(R.core_nufft, p.u_dx, p.v_dy, vr, p.vis_i, p.vis_std, 64, 64, 1000, 1e-5,
                            lam1, 0.0, lamt, cinit, nonneg_flag=1)
        dx = max(dx, np.linalg.norm(x2 - out["x_1000"]) / np.linalg.norm(out["x_1000"]))
        dc = max(dc, abs(r2.finalcost - out["res_1000"][RES_KEYS.index("finalcost")]) /
                 out["res_1000"][RES_KEYS.index("finalcost")])
    out["envelope_x_1000"] = dx
    out["envelope_cost_1000"] = dc
    # variants (short runs)
    box = (np.arange(64 * 64) % 64 >= 8).astype(np.float32)
    out["box"] = box
    var = {
        "real": dict(nonneg_flag=0),
        "box": dict(nonneg_flag=1, box_flag=1, cl_box=box),
        "warm": dict(nonneg_flag=1, xinit=p.sky.ravel() * 0.5),
        "tv": dict(nonneg_flag=1, lam_tv=5e-3 * lam1, lam_tsv=0.0),
        "tv_real": dict(nonneg_flag=0, lam_tv=5e-3 * lam1, lam_tsv=0.0),
        "l1only": dict(nonneg_flag=1, lam_tsv=0.0),
        "stop": dict(nonneg_flag=1, eps=300.0, maxiter=1000),
        "zero": dict(nonneg_flag=1, lam1=10 * np.abs(g0).max(), maxiter=200),
        "maxiter0": dict(nonneg_flag=1, maxiter=0),
        "badflag": dict(nonneg_flag=2),
    }
    for name, kw in var.items():
        kw = dict(kw)
        ltv = kw.pop("lam_tv", 0.0)
        lts = kw.pop("lam_tsv", lamt)
        eps = kw.pop("eps", 1e-5)
        l1 = kw.pop("lam1", lam1)
        mi = kw.pop("maxiter", 60 if ltv else 150)
        x, res = quiet_call(R.core_nufft, *args, mi, eps, l1, ltv, lts, cinit, **kw)
        out[f"var_{name}_x"] = x
        out[f"var_{name}_res"] = res_arr(res)
        out[f"var_{name}_cfg"] = np.array([mi, ltv, lts, kw.get("nonneg_flag", 1), kw.get("box_flag", 0),
                                           1.0 if "xinit" in kw else 0.0, eps, l1])
    np.savez_compressed(os.path.join(HERE, "c0_nufft.npz"), **out)


def make_c1():
    p = synth.fft_problem(nx=128, n_cells=3000, seed=1)
    op = O.FftOperator(p.u_idx, p.v_idx, p.y_r, p.y_i, p.noise_stdev, 128, 128)
    g0 = op.grad(op.f_part(np.zeros(128 * 128))[1])
    lam1 = 1e-2 * np.abs(g0).max()
    lamtv = 5e-3 * lam1
    lamtsv = 1e-3 * lam1
    # Lipschitz of the FFT variant: mask^2 / 2 at most (half-spectrum weights)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(128 * 128)
    lip = 0.0
    for _ in range(30):
        x /= np.linalg.norm(x)
        _, r = op.f_part(x)
        # gradient of F at x with y = 0 is -(dF); use the operator on -A x
        y = op.grad(-(op.yf_h - r))
        lip = float(x @ y)
        x = y
    cinit = abs(lip)
    out = dict(u_idx=p.u_idx, v_idx=p.v_idx, y_r=p.y_r, y_i=p.y_i, noise=p.noise_stdev,
               sky=p.sky.ravel(), lam1=lam1, lamtv=lamtv, lamtsv=lamtsv, cinit=cinit)
    args = (p.u_idx, p.v_idx, p.y_r, p.y_i, p.noise_stdev, 128, 128)
    x, res = quiet_call(R.core_fft, *args, 300, 1e-5, lam1, 0.0, lamtsv, cinit, nonneg_flag=1)
    out["tsv_x"], out["tsv_res"] = x, res_arr(res)
    x, res = quiet_call(R.core_fft, *args, 40, 1e-5, lam1, lamtv, 0.0, cinit, nonneg_flag=1)
    out["tv100_x"], out["tv100_res"] = x, res_arr(res)
    x, res = quiet_call(R.core_fft, *args, 40, 1e-5, lam1, lamtv, 0.0, cinit, nonneg_flag=1, fgp50=True)
    out["tv50_x"], out["tv50_res"] = x, res_arr(res)
    x, res = quiet_call(R.core_fft, *args, 40, 1e-5, lam1, lamtv, 0.0, cinit, nonneg_flag=0)
    out["tvreal_x"], out["tvreal_res"] = x, res_arr(res)
    # FGP alone
    b = p.sky.ravel() + 1e-4 * rng.standard_normal(128 * 128)
    out["fgp_b"] = b
    out["fgp_nonneg"] = R.fgp(128, 128, b, 0.0, 2e-4, 100, True)
    out["fgp_l1"] = R.fgp(128, 128, b, 1e-5, 2e-4, 100, False)
    np.savez_compressed(os.path.join(HERE, "c1_fft.npz"), **out)


def make_c1long():
    """Config 1 run long: the TV form with FGP 50 (the reference built with
    FGPITER 50) for 1000 iterations with the stopping rule off, and the
    reference's own spread under a 1e-15 change of one visibility."""
    g = np.load(os.path.join(HERE, "c1_fft.npz"))
    args = (g["u_idx"], g["v_idx"], g["y_r"], g["y_i"], g["noise"], 128, 128)
    lam1, lamtv, cinit = float(g["lam1"]), float(g["lamtv"]), float(g["cinit"])
    x, res = quiet_call(R.core_fft, *args, 1000, 0.0, lam1, lamtv, 0.0, cinit, nonneg_flag=1, fgp50=True)
    yr = g["y_r"].copy()
    yr[0] *= 1 + 1e-15
    x2, res2 = quiet_call(R.core_fft, g["u_idx"], g["v_idx"], yr, g["y_i"], g["noise"], 128, 128, 1000, 0.0, lam1,
                          lamtv, 0.0, cinit, nonneg_flag=1, fgp50=True)
    out = dict(x=x, res=res_arr(res), iters=1000,
               envelope_x=float(np.linalg.norm(x2 - x) / np.linalg.norm(x)),
               envelope_cost=abs(res2.finalcost - res.finalcost) / res.finalcost)
    np.savez_compressed(os.path.join(HERE, "c1_tv50_1000.npz"), **out)
    print("c1long", res.ITER, res.finalcost, out["envelope_x"], out["envelope_cost"])


def make_c2small():
    p = synth.dft_problem(nx=16, n_stations=6, n_hours=10, seed=2, m_vis=150)
    A = np.asarray(p.A)
    op = O.DftOperator(p.y, A)
    g0 = op.grad(p.y)
    lam1 = 1e-2 * np.abs(g0).max()
    cinit = float(np.linalg.norm(A, 2) ** 2)
    out = dict(y=p.y, A=A, lam1=lam1, cinit=cinit, nx=16)
    x, res, resid = quiet_call(R.core_dft, p.y, A, 16, 16, 300, 1e-6, lam1, 0.0, 1e-3 * lam1, cinit,
                               nonneg_flag=1)
    out["tsv_x"], out["tsv_res"], out["tsv_resid"] = x, res_arr(res), resid
    x, res, resid = quiet_call(R.core_dft, p.y, A, 16, 16, 40, 1e-6, lam1, 5e-3 * lam1, 0.0, cinit,
                               nonneg_flag=1)
    out["tv_x"], out["tv_res"], out["tv_resid"] = x, res_arr(res), resid
    np.savez_compressed(os.path.join(HERE, "c2_dft_small.npz"), **out)


if __name__ == "__main__":
    which = sys.argv[1:] or ["c0", "c1", "c2", "c1long"]
    if "c0" in which:
        make_c0()
    if "c1" in which:
        make_c1()
    if "c2" in which:
        make_c2small()
    if "c1long" in which:
        make_c1long()
    print("golden fixtures written to", HERE)
