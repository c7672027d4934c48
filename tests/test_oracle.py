"""The oracle (numpy restatement) pinned against the reference's outputs.

The golden fixtures hold outputs of the reference C solvers compiled
unchanged (tests/golden/make_golden.py).  These tests need no GPU.
"""
import os

import numpy as np
import pytest

from conftest import REFERENCE_C, rel, res_dict
from oracle import mfista_oracle as O


def _solve_c0(c0, maxiter, eps=1e-5, lam1=None, ltv=0.0, lts=None, nonneg=1, box_flag=0,
              cl_box=None, xinit=None):
    lam1 = float(c0["lam1"]) if lam1 is None else lam1
    lts = float(c0["lamt"]) if lts is None else lts
    x0 = np.zeros(64 * 64) if xinit is None else xinit
    return O.imaging_core_nufft(c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"], 64, 64,
                                maxiter, eps, lam1, ltv, lts, float(c0["cinit"]), x0, nonneg,
                                box_flag, cl_box)


def test_nufft_forward_matches_reference(c0):
    plan = O.NufftPlan(c0["u"], c0["v"], 64, 64)
    fr, fi = plan.forward(c0["sky"])
    assert rel(fr + 1j * fi, c0["fwd_r"] + 1j * c0["fwd_i"]) < 1e-13


def test_nufft_adjoint_matches_reference(c0):
    plan = O.NufftPlan(c0["u"], c0["v"], 64, 64)
    x = plan.adjoint(c0["adj_in_r"], c0["adj_in_i"])
    assert rel(x, c0["adj_out"]) < 1e-13


def test_nufft_forward_is_the_dft(c0):
    """Known answer: the gridding approximates V = sum x exp(+i(u(i-Nx/2)+v(j-Ny/2)))."""
    from sparseimaging_b200 import synth
    plan = O.NufftPlan(c0["u"], c0["v"], 64, 64)
    sky = c0["sky"].reshape(64, 64)
    fr, fi = plan.forward(sky.ravel())
    v = synth.dft_vis(sky, c0["u"], c0["v"])
    assert rel(fr + 1j * fi, v) < 1e-11


def test_nufft_adjointness(c0):
    plan = O.NufftPlan(c0["u"], c0["v"], 64, 64)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(64 * 64)
    a, b = rng.standard_normal(c0["u"].size), rng.standard_normal(c0["u"].size)
    fr, fi = plan.forward(x)
    lhs = fr @ a + fi @ b
    rhs = x @ plan.adjoint(a, b)
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


@pytest.mark.parametrize("name", ["real", "box", "warm", "l1only", "zero", "maxiter0", "badflag"])
def test_oracle_nufft_variants(c0, name):
    cfg = c0[f"var_{name}_cfg"]
    mi, ltv, lts, nn, bf, warm, eps, l1 = cfg
    x0 = c0["sky"] * 0.5 if warm else None
    x, res = _solve_c0(c0, int(mi), eps=eps, lam1=l1, ltv=ltv, lts=lts, nonneg=int(nn),
                       box_flag=int(bf), cl_box=c0["box"] if bf else None, xinit=x0)
    gold = res_dict(c0[f"var_{name}_res"])
    assert res["ITER"] == gold["ITER"]
    assert rel(x, c0[f"var_{name}_x"]) < 1e-7
    assert abs(res["finalcost"] - gold["finalcost"]) <= 1e-10 * abs(gold["finalcost"])
    assert res["N_active"] == gold["N_active"]
    assert res["M"] == gold["M"]


def test_oracle_nufft_tv(c0):
    cfg = c0["var_tv_cfg"]
    x, res = _solve_c0(c0, int(cfg[0]), ltv=cfg[1], lts=0.0)
    gold = res_dict(c0["var_tv_res"])
    assert rel(x, c0["var_tv_x"]) < 1e-7
    assert abs(res["finalcost"] - gold["finalcost"]) <= 1e-10 * gold["finalcost"]


def test_oracle_nufft_stop_rule(c0):
    cfg = c0["var_stop_cfg"]
    x, res = _solve_c0(c0, int(cfg[0]), eps=cfg[6])
    gold = res_dict(c0["var_stop_res"])
    assert res["ITER"] == gold["ITER"] < int(cfg[0])
    assert rel(x, c0["var_stop_x"]) < 1e-7


def test_oracle_fft_variant(c1):
    args = (c1["u_idx"], c1["v_idx"], c1["y_r"], c1["y_i"], c1["noise"], 128, 128)
    lam1, cinit = float(c1["lam1"]), float(c1["cinit"])
    x, res = O.imaging_core_fft(*args, 300, 1e-5, lam1, 0.0, float(c1["lamtsv"]), cinit,
                                np.zeros(128 * 128), 1)
    g = res_dict(c1["tsv_res"])
    assert rel(x, c1["tsv_x"]) < 1e-7
    assert abs(res["finalcost"] - g["finalcost"]) <= 1e-10 * g["finalcost"]
    for key, it in (("tv100", 100), ("tv50", 50)):
        x, res = O.imaging_core_fft(*args, 40, 1e-5, lam1, float(c1["lamtv"]), 0.0, cinit,
                                    np.zeros(128 * 128), 1, fgp_iter=it)
        g = res_dict(c1[f"{key}_res"])
        assert rel(x, c1[f"{key}_x"]) < 1e-7
        assert abs(res["finalcost"] - g["finalcost"]) <= 1e-10 * g["finalcost"]


def test_oracle_fgp(c1):
    b = c1["fgp_b"]
    assert rel(O.fgp(128, 128, b, 0.0, 2e-4, 100, True), c1["fgp_nonneg"]) < 1e-12
    assert rel(O.fgp(128, 128, b, 1e-5, 2e-4, 100, False), c1["fgp_l1"]) < 1e-12


def test_oracle_dft_variant(c2):
    lam1, cinit, nx = float(c2["lam1"]), float(c2["cinit"]), int(c2["nx"])
    x, res = O.imaging_core_dft(c2["y"], c2["A"], nx, nx, 300, 1e-6, lam1, 0.0, 1e-3 * lam1, cinit,
                                np.zeros(nx * nx), 1)
    g = res_dict(c2["tsv_res"])
    assert res["ITER"] == g["ITER"]
    assert rel(x, c2["tsv_x"]) < 1e-7
    assert abs(res["finalcost"] - g["finalcost"]) <= 1e-10 * g["finalcost"]
    assert rel(res["residual"], c2["tsv_resid"]) < 1e-7
    x, res = O.imaging_core_dft(c2["y"], c2["A"], nx, nx, 40, 1e-6, lam1, 5e-3 * lam1, 0.0, cinit,
                                np.zeros(nx * nx), 1)
    assert rel(x, c2["tv_x"]) < 1e-7


@pytest.mark.slow
def test_oracle_trajectory_400(c0):
    """400 iterations of config 0: the oracle follows the reference to 1e-7."""
    x, res = _solve_c0(c0, 400)
    g = res_dict(c0["res_400"])
    assert rel(x, c0["x_400"]) < 1e-7
    assert abs(res["finalcost"] - g["finalcost"]) <= 1e-10 * g["finalcost"]


def test_regularisers_match_reference_formulas(c0):
    """TSV / TV / d_TSV on a non-square view (NX != NY) against loops written
    from c/mfista_tools.c:145-186 and c/mfista_TV_lib.c:30-46."""
    rng = np.random.default_rng(3)
    NX, NY = 7, 5
    x = rng.standard_normal(NX * NY)
    tsv = sum((x[NX * j + i] - x[NX * j + i + 1]) ** 2 for j in range(NY) for i in range(NX - 1))
    tsv += sum((x[NX * j + i] - x[NX * (j + 1) + i]) ** 2 for j in range(NY - 1) for i in range(NX))
    assert abs(O.tsv(NX, NY, x) - tsv) < 1e-12
    tv = sum(np.sqrt((x[NX * j + i] - x[NX * j + i + 1]) ** 2 + (x[NX * j + i] - x[NX * (j + 1) + i]) ** 2)
             for i in range(NX - 1) for j in range(NY - 1))
    tv += sum(abs(x[NX * (NY - 1) + i] - x[NX * (NY - 1) + i + 1]) for i in range(NX - 1))
    tv += sum(abs(x[NX * j + NX - 1] - x[NX * (j + 1) + NX - 1]) for j in range(NY - 1))
    assert abs(O.tv(NX, NY, x) - tv) < 1e-12
    d = np.zeros(NX * NY)
    for j in range(NY):
        for i in range(NX):
            f = NX * j + i
            v = 2 * (x[f] - x[f + 1]) if i < NX - 1 else 0.0
            if i >= 1:
                v += 2 * (x[f] - x[f - 1])
            if j < NY - 1:
                v += 2 * (x[f] - x[f + NX])
            if j >= 1:
                v += 2 * (x[f] - x[f - NX])
            d[f] = v
    assert np.abs(O.d_tsv(NX, NY, x) - d).max() < 1e-12


@pytest.mark.skipif(not os.path.isdir(REFERENCE_C), reason="reference sources not present")
def test_oracle_on_reference_fixture_file():
    """The reference's own sample data (c/nufft_data.txt, Nx = 200, a
    non-power-of-two padded grid of 400): oracle operators vs the compiled
    reference."""
    from oracle import ref_ctypes as R
    if not R.available():
        pytest.skip("oracle/_ref not built")
    rows = np.loadtxt(os.path.join(REFERENCE_C, "nufft_data.txt"), delimiter=",", skiprows=5)
    u, v = rows[:, 0], rows[:, 1]
    plan = O.NufftPlan(u, v, 200, 200)
    ref = R.RefNufft(u, v, 200, 200)
    rng = np.random.default_rng(0)
    x = rng.random(200 * 200)
    fr, fi = plan.forward(x)
    gr, gi = ref.forward(x)
    assert rel(fr + 1j * fi, gr + 1j * gi) < 1e-12
    a, b = rng.standard_normal(u.size), rng.standard_normal(u.size)
    assert rel(plan.adjoint(a, b), ref.adjoint(a, b)) < 1e-12
    ref.close()
