"""Drop-in FP64 solves on the GPU against the reference's own outputs.

Parity bars (FP64 plain method):
  * trajectories the reference itself reproduces under 1-ulp input
    perturbations (<= 400 iterations on config 0, every short variant):
    xout within 1e-7 relative L2 and the final objective within 1e-10
    relative, ITER and N_active equal;
  * config 0 at its full 1000 iterations, where the reference's own output
    moves by ~1.5e-4 (xout) / ~2e-8 (objective) under a 1e-15 perturbation
    of one visibility (stored as envelope_*_1000 in the fixture): within 10x
    that envelope.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel, res_dict

pytestmark = pytest.mark.gpu


def _c0_solve(si, c0, maxiter, eps=1e-5, lam1=None, ltv=0.0, lts=None, nonneg=1, box_flag=0,
              cl_box=None, xinit=None):
    lam1 = float(c0["lam1"]) if lam1 is None else lam1
    lts = float(c0["lamt"]) if lts is None else lts
    return si.imaging_core_nufft(c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"], 64, 64,
                                 maxiter, eps, lam1, ltv, lts, float(c0["cinit"]), xinit=xinit,
                                 nonneg_flag=nonneg, box_flag=box_flag, cl_box=cl_box)


def _check_result(res, gold, x, gx, xtol=1e-7, ctol=1e-10):
    assert res["ITER"] == gold["ITER"]
    assert res["M"] == gold["M"] and res["N"] == gold["N"]
    assert res["NX"] == gold["NX"] and res["NY"] == gold["NY"]
    assert res["nonneg"] == gold["nonneg"] and res["maxiter"] == gold["maxiter"]
    assert rel(x, gx) <= xtol
    assert abs(res["finalcost"] - gold["finalcost"]) <= ctol * abs(gold["finalcost"])
    assert abs(res["sq_error"] - gold["sq_error"]) <= 1e-8 * abs(gold["sq_error"]) + 1e-12
    assert abs(res["l1cost"] - gold["l1cost"]) <= 1e-7 * abs(gold["l1cost"]) + 1e-300
    assert abs(res["Lip_const"] - gold["Lip_const"]) <= 1e-9 * abs(gold["Lip_const"])


def test_nufft_400_iterations_match_reference(gpulib, c0):
    x, res = _c0_solve(gpulib, c0, 400)
    gold = res_dict(c0["res_400"])
    _check_result(res, gold, x, c0["x_400"])
    assert res["N_active"] == gold["N_active"]
    assert abs(res["tsvcost"] - gold["tsvcost"]) <= 1e-8 * gold["tsvcost"]
    assert abs(res["mean_sq_error"] - gold["mean_sq_error"]) <= 1e-8 * gold["mean_sq_error"]


def test_nufft_config0_within_reference_envelope(gpulib, c0):
    x, res = _c0_solve(gpulib, c0, 1000)
    gold = res_dict(c0["res_1000"])
    assert res["ITER"] == gold["ITER"] == 1000
    env_x, env_c = float(c0["envelope_x_1000"]), float(c0["envelope_cost_1000"])
    assert rel(x, c0["x_1000"]) <= 10 * env_x
    assert abs(res["finalcost"] - gold["finalcost"]) <= 10 * env_c * gold["finalcost"]


@pytest.mark.parametrize("name", ["real", "box", "warm", "l1only", "tv", "tv_real", "stop", "zero",
                                  "maxiter0", "badflag"])
def test_nufft_variants_match_reference(gpulib, c0, name):
    mi, ltv, lts, nn, bf, warm, eps, l1 = c0[f"var_{name}_cfg"]
    x0 = c0["sky"] * 0.5 if warm else None
    x, res = _c0_solve(gpulib, c0, int(mi), eps=eps, lam1=l1, ltv=ltv, lts=lts, nonneg=int(nn),
                       box_flag=int(bf), cl_box=c0["box"] if bf else None, xinit=x0)
    gold = res_dict(c0[f"var_{name}_res"])
    _check_result(res, gold, x, c0[f"var_{name}_x"])
    assert res["N_active"] == gold["N_active"]


def test_nufft_both_regularisers_is_an_error(gpulib, c0):
    """Reference: prints and returns with RESULT untouched (:938-941)."""
    r = gpulib.RESULT()
    r.ITER = -7
    xo = np.full(64 * 64, 3.0)
    box = np.ones(64 * 64, np.float32)
    gpulib.mfista_imaging_core_nufft(c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"],
                                     c0["u"].size, 64, 64, 10, 1e-5, 1.0, 1.0, 1.0, 1e9,
                                     np.zeros(64 * 64), xo, 1, 0, box, r)
    assert gpulib.last_status() == 4
    assert r.ITER == -7 and np.all(xo == 3.0)


def test_fft_variant_tsv(gpulib, c1):
    args = (c1["u_idx"], c1["v_idx"], c1["y_r"], c1["y_i"], c1["noise"], 128, 128)
    x, res = gpulib.imaging_core_fft(*args, 300, 1e-5, float(c1["lam1"]), 0.0, float(c1["lamtsv"]),
                                     float(c1["cinit"]))
    gold = res_dict(c1["tsv_res"])
    _check_result(res, gold, x, c1["tsv_x"])


@pytest.mark.parametrize("key,fgp,nonneg", [("tv100", 100, 1), ("tv50", 50, 1), ("tvreal", 100, 0)])
def test_fft_variant_tv(gpulib, c1, key, fgp, nonneg):
    args = (c1["u_idx"], c1["v_idx"], c1["y_r"], c1["y_i"], c1["noise"], 128, 128)
    old = gpulib.set_fgp_iter(fgp)
    try:
        x, res = gpulib.imaging_core_fft(*args, 40, 1e-5, float(c1["lam1"]), float(c1["lamtv"]), 0.0,
                                         float(c1["cinit"]), nonneg_flag=nonneg)
    finally:
        gpulib.set_fgp_iter(old)
    gold = res_dict(c1[f"{key}_res"])
    _check_result(res, gold, x, c1[f"{key}_x"])
    assert abs(res["tvcost"] - gold["tvcost"]) <= 1e-8 * gold["tvcost"]


def test_dft_variant_tsv(gpulib, c2):
    nx = int(c2["nx"])
    lam1, cinit = float(c2["lam1"]), float(c2["cinit"])
    x, res = gpulib.imaging_core_dft(c2["y"], c2["A"], nx, nx, 300, 1e-6, lam1, 0.0, 1e-3 * lam1, cinit)
    gold = res_dict(c2["tsv_res"])
    _check_result(res, gold, x, c2["tsv_x"])
    assert rel(res["residual"], c2["tsv_resid"]) < 1e-7


def test_dft_variant_tv(gpulib, c2):
    nx = int(c2["nx"])
    lam1, cinit = float(c2["lam1"]), float(c2["cinit"])
    x, res = gpulib.imaging_core_dft(c2["y"], c2["A"], nx, nx, 40, 1e-6, lam1, 5e-3 * lam1, 0.0, cinit)
    gold = res_dict(c2["tv_res"])
    _check_result(res, gold, x, c2["tv_x"])


def test_dft_raw_entry_point_allocates_residual(gpulib, c2):
    nx = int(c2["nx"])
    A = np.asfortranarray(c2["A"])
    m, n = A.shape
    r = gpulib.RESULT()
    xo = np.zeros(n)
    box = np.ones(n, np.float32)
    gpulib.mfista_imaging_core_dft(np.ascontiguousarray(c2["y"]), A, C.c_int(m), C.c_int(n), nx, nx, 300,
                                   1e-6, float(c2["lam1"]), 0.0, 1e-3 * float(c2["lam1"]),
                                   float(c2["cinit"]), np.zeros(n), xo, 1, 0, 0, box, r)
    assert gpulib.last_status() == 0
    assert bool(r.residual)
    resid = np.ctypeslib.as_array(r.residual, shape=(m,)).copy()
    assert rel(resid, c2["tsv_resid"]) < 1e-7
    C.CDLL(None).free(C.cast(r.residual, C.c_void_p))


def test_dft_batch_gemm_matches_reference(gpulib, c2):
    """Three problems through the batched GEMM path; the one with the golden
    parameters matches the reference's output."""
    nx = int(c2["nx"])
    lam1, cinit = float(c2["lam1"]), float(c2["cinit"])
    probs = [dict(lambda_l1=lam1 * s, lambda_tsv=1e-3 * lam1 * s, cinit=cinit, maxiter=300, nonneg_flag=1)
             for s in (0.5, 1.0, 3.0)]
    X, R = gpulib.dft_batch(c2["y"], c2["A"], nx, nx, probs, 1e-6)
    gold = res_dict(c2["tsv_res"])
    assert R[1]["ITER"] == gold["ITER"]
    assert rel(X[1], c2["tsv_x"]) < 1e-7
    assert abs(R[1]["finalcost"] - gold["finalcost"]) <= 1e-10 * gold["finalcost"]
    for b in (0, 2):
        x, r = gpulib.imaging_core_dft(c2["y"], c2["A"], nx, nx, 300, 1e-6, probs[b]["lambda_l1"], 0.0,
                                       probs[b]["lambda_tsv"], cinit)
        assert R[b]["ITER"] == r["ITER"]
        assert rel(X[b], x) < 1e-7
