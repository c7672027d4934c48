"""Full solves on the reference's own sample data against the reference.

Fixtures (tests/golden/make_refdata_golden.py, the reference C compiled
here): c/nufft_data.txt (200 x 200, M = 7648) with the parameter set of
matlab/testdata4nufft.mat, and c/fft_data.txt (128 x 128, M = 6590) as an
L1+TSV and an L1+TV problem with matlab/test_algorithm.m's parameters, each
run through mfista_imaging_core_* to the reference's own stopping rule.

The FFT solves are stable under 1-ulp input changes (the reference's own
envelope is ~1e-14), so the GPU must match them as the contract states:
xout to 1e-7, the objective to 1e-10, the iteration count exactly.  The
NUFFT solve runs 2365 iterations and is chaotic from about iteration 60 on:
one visibility changed by 1e-15 moves the reference's own xout by 1e-7
after 60 iterations, 1.4e-3 after 100 and 3.7e-3 (and its iteration count
by 17) at the end.  The GPU is held to the first 30 iterations at the
contract's tolerances and, over the full run, to a few times that envelope.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel, res_dict

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nu():
    return np.load(os.path.join(GOLDEN, "refdata_nufft.npz"))


@pytest.fixture(scope="module")
def ff():
    return np.load(os.path.join(GOLDEN, "refdata_fft.npz"))


def _nufft(gpulib, g, maxiter):
    return gpulib.imaging_core_nufft(g["u"], g["v"], g["vis_r"], g["vis_i"], g["vis_std"], int(g["nx"]),
                                     int(g["ny"]), maxiter, float(g["eps"]), float(g["lam1"]), 0.0,
                                     float(g["lamtsv"]), float(g["cinit"]), nonneg_flag=1)


def test_nufft_sample_data_30_iterations(gpulib, nu):
    x, r = _nufft(gpulib, nu, 30)
    gold = res_dict(nu["short_res"])
    assert r["ITER"] == gold["ITER"] == 30
    assert rel(x, nu["short_x"]) < 1e-7
    assert abs(r["finalcost"] - gold["finalcost"]) <= 1e-10 * gold["finalcost"]
    assert r["N_active"] == gold["N_active"] and r["M"] == gold["M"]


def test_nufft_sample_data_full_solve(gpulib, nu):
    """eps 1e-3, maxiter 5000: within 3x the reference's own 1-ulp envelope
    (xout, objective) and 3 % of its iteration count."""
    x, r = _nufft(gpulib, nu, int(nu["maxiter"]))
    gold = res_dict(nu["full_res"])
    ex, ec = float(nu["full_envelope_x"]), float(nu["full_envelope_cost"])
    assert abs(r["ITER"] - gold["ITER"]) <= 0.03 * gold["ITER"]
    assert rel(x, nu["full_x"]) < max(1e-7, 3 * ex)
    assert abs(r["finalcost"] - gold["finalcost"]) <= max(1e-10, 3 * ec) * gold["finalcost"]


@pytest.mark.parametrize("form", ["tsv", "tv"])
def test_fft_sample_data_full_solve(gpulib, ff, form):
    lam2 = float(ff["lam2"])
    ltv, lts = (0.0, lam2) if form == "tsv" else (lam2, 0.0)
    x, r = gpulib.imaging_core_fft(ff["u_idx"], ff["v_idx"], ff["y_r"], ff["y_i"], ff["noise"], int(ff["nx"]),
                                   int(ff["ny"]), int(ff["maxiter"]), float(ff["eps"]), float(ff["lam1"]), ltv,
                                   lts, float(ff["cinit"]), nonneg_flag=1)
    gold = res_dict(ff[f"{form}_res"])
    assert r["ITER"] == gold["ITER"]
    assert rel(x, ff[f"{form}_x"]) < 1e-7
    assert abs(r["finalcost"] - gold["finalcost"]) <= 1e-10 * gold["finalcost"]
    assert r["N_active"] == gold["N_active"]
