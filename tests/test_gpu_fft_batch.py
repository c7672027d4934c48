"""Batched FFT (gridded) variant, FP64 and the corrected FP32 form.

An FP64 batch reproduces the drop-in mfista_imaging_core_fft problem by
problem (the kernels never mix problems).  The FP32 form (FP32 FFTs and FGP
stencils, forward spectrum corrected by the exact FP64 spectrum of an anchor
image, FP64 objective and backtracking) is held to the FP64 objective.
Inputs: the config-1 fixture (128 x 128, 3000 cells with their Hermitian
partners, L1+TV with FGP 50 and L1+TSV), made from the reference by
tests/golden/make_golden.py.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel, res_dict

pytestmark = pytest.mark.gpu


def _data(c1):
    return (c1["u_idx"], c1["v_idx"], c1["y_r"], c1["y_i"], c1["noise"], 128, 128)


def _tv_problems(c1, scales, maxiter):
    lam1, ltv = float(c1["lam1"]), float(c1["lamtv"])
    return [dict(lambda_l1=lam1 * s, lambda_tv=ltv * s, cinit=float(c1["cinit"]), maxiter=maxiter, nonneg_flag=1)
            for s in scales]


def _tsv_problems(c1, scales, maxiter):
    lam1, lts = float(c1["lam1"]), float(c1["lamtsv"])
    return [dict(lambda_l1=lam1 * s, lambda_tsv=lts * s, cinit=float(c1["cinit"]), maxiter=maxiter, nonneg_flag=1)
            for s in scales]


def test_fp64_tv_batch_equals_single(gpulib, c1):
    probs = _tv_problems(c1, [0.5, 1.0, 2.0], 30)
    old = gpulib.set_fgp_iter(50)
    try:
        singles = [gpulib.imaging_core_fft(*_data(c1), 30, 1e-5, p["lambda_l1"], p["lambda_tv"], 0.0, p["cinit"])
                   for p in probs]
    finally:
        gpulib.set_fgp_iter(old)
    X, R = gpulib.fft_batch(*_data(c1), probs, 1e-5, fgp_iter=50)
    for b, (x, r) in enumerate(singles):
        assert R[b]["ITER"] == r["ITER"]
        assert rel(X[b], x) < 1e-13
        assert abs(R[b]["finalcost"] - r["finalcost"]) <= 1e-13 * r["finalcost"]


def test_fp64_batch_matches_reference_fgp50(gpulib, c1):
    """Problem 0 of a batch is the config-1 TV solve with FGP 50, checked
    against the reference built with FGPITER 50 (40 iterations)."""
    probs = _tv_problems(c1, [1.0, 3.0], 40)
    X, R = gpulib.fft_batch(*_data(c1), probs, 1e-5, fgp_iter=50)
    gold = res_dict(c1["tv50_res"])
    assert R[0]["ITER"] == gold["ITER"]
    assert rel(X[0], c1["tv50_x"]) < 1e-7
    assert abs(R[0]["finalcost"] - gold["finalcost"]) <= 1e-10 * gold["finalcost"]


@pytest.mark.parametrize("form", ["tv", "tsv"])
def test_fp32_form_reaches_fp64_objective(gpulib, c1, form):
    """FP32 operators with the FP64 anchor correction reach the objective of
    the FP64 solve to 1e-6 relative, in about the FP64 iteration count."""
    mk = _tv_problems if form == "tv" else _tsv_problems
    probs = mk(c1, [0.5, 1.0, 2.0], 300)
    X64, R64 = gpulib.fft_batch(*_data(c1), probs, 0.0, fgp_iter=50)
    targets = [r["finalcost"] * (1 + 1e-6) for r in R64]
    for p, t in zip(probs, targets):
        p["target_cost"] = t
        p["maxiter"] = 1200
    X32, R32 = gpulib.fft_batch(*_data(c1), probs, 0.0, fgp_iter=50, precision=gpulib.FP32)
    for b, (r, t) in enumerate(zip(R32, targets)):
        assert r["finalcost"] <= t, (b, r["finalcost"], t)
        assert r["ITER"] < 1200
        assert rel(X32[b], X64[b]) < 2e-2


def test_fp32_short_run_tracks_fp64(gpulib, c1):
    """20 iterations of the TV form: the FP32 form's objective within 1e-6
    of the FP64 one (the corrected forward spectrum is FP64 up to the FP32
    error of the departure from the anchor)."""
    probs = _tv_problems(c1, [1.0], 20)
    _, R64 = gpulib.fft_batch(*_data(c1), probs, 0.0, fgp_iter=50)
    _, R32 = gpulib.fft_batch(*_data(c1), probs, 0.0, fgp_iter=50, precision=gpulib.FP32)
    assert R32[0]["ITER"] == R64[0]["ITER"] == 20
    assert abs(R32[0]["finalcost"] - R64[0]["finalcost"]) <= 1e-6 * R64[0]["finalcost"]


def test_config1_1000_iterations_both_forms(gpulib, c1):
    """Config 1 (TV form, FGP 50) for 1000 iterations, stopping rule off,
    against the reference built with FGPITER 50 (tests/golden/c1_tv50_1000.npz;
    its own spread under a 1e-15 input change is ~2e-14, so the run is on
    one trajectory): the FP64 solve to the contract's tolerances, the FP32
    form's objective to 1e-6 of the reference's."""
    ref = np.load(os.path.join(GOLDEN, "c1_tv50_1000.npz"))
    gold = res_dict(ref["res"])
    probs = _tv_problems(c1, [1.0], 1000)
    X64, R64 = gpulib.fft_batch(*_data(c1), probs, 0.0, fgp_iter=50)
    assert R64[0]["ITER"] == 1000
    assert rel(X64[0], ref["x"]) < 1e-7
    assert abs(R64[0]["finalcost"] - gold["finalcost"]) <= 1e-10 * gold["finalcost"]
    X32, R32 = gpulib.fft_batch(*_data(c1), probs, 0.0, fgp_iter=50, precision=gpulib.FP32)
    assert abs(R32[0]["finalcost"] - gold["finalcost"]) <= 1e-6 * gold["finalcost"]
    assert rel(X32[0], ref["x"]) < 1e-2


def test_fft_batch_rejects_bad_arguments(gpulib, c1):
    probs = _tv_problems(c1, [1.0], 10)
    with pytest.raises(gpulib.MfistaError):
        gpulib.fft_batch(*_data(c1), probs, 1e-5, precision=gpulib.BF16X3)
    p2 = [dict(probs[0]), dict(probs[0])]
    p2[1]["lambda_tv"] = 0.0
    p2[1]["lambda_tsv"] = 1.0
    with pytest.raises(gpulib.MfistaError):
        gpulib.fft_batch(*_data(c1), p2, 1e-5)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_fgp_profile_times_the_prox(gpulib, prec):
    p = gpulib.FP64 if prec == "fp64" else gpulib.FP32
    ms, by = gpulib.fgp_profile(128, 128, 4, 50, precision=p, reps=3)
    assert ms > 0
    assert by == 24.0 * 4 * 128 * 128
