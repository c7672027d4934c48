"""Launch shapes and the autotuner of the batched plan.

Row/column FFT shapes must leave a solve bit-identical; the interpolation
and spreading shapes regroup sums, so FP64 results may move by rounding only
(1e-10 relative on ~150 iterations of config 0, far inside the parity bars).
"""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


def _plan(si, c0, precision=None, B=4):
    precision = si.FP64 if precision is None else precision
    lam1 = float(c0["lam1"])
    probs = [dict(lambda_l1=lam1 * s, lambda_tsv=lam1 * 1e-3 * s, cinit=float(c0["cinit"]), maxiter=150,
                  nonneg_flag=1) for s in np.geomspace(0.2, 5.0, B)]
    plan = si.Plan(c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"], 64, 64, B, precision=precision)
    return plan, probs


def _solve(plan, probs):
    plan.set_problems(probs, 1e-5)
    plan.run()
    return plan.fetch()


def test_row_and_column_shapes_are_bit_identical(gpulib, c0):
    plan, probs = _plan(gpulib, c0)
    X0, R0 = _solve(plan, probs)
    base = plan.shapes()
    assert base["rows_per_cta"] > 0 and base["cols_per_cta"] > 0
    for rows, cols in [(1, 1), (2, 4), (16, 16)]:
        plan.set_shapes(rows_per_cta=rows, cols_per_cta=cols)
        assert plan.shapes()["rows_per_cta"] == rows and plan.shapes()["cols_per_cta"] == cols
        X, R = _solve(plan, probs)
        assert np.array_equal(X, X0)
        assert [r["ITER"] for r in R] == [r["ITER"] for r in R0]
        assert [r["finalcost"] for r in R] == [r["finalcost"] for r in R0]
    plan.close()


def test_interp_and_spread_shapes_move_results_by_rounding_only(gpulib, c0):
    plan, probs = _plan(gpulib, c0)
    X0, R0 = _solve(plan, probs)
    for ppw, cl in [(1, 1), (4, 2), (16, 4)]:
        plan.set_shapes(interp_ppw=ppw, spread_cluster=cl)
        sh = plan.shapes()
        assert sh["interp_ppw"] == ppw and sh["spread_cluster"] == cl
        X, R = _solve(plan, probs)
        for b in range(len(probs)):
            assert R[b]["ITER"] == R0[b]["ITER"]
            assert rel(X[b], X0[b]) < 1e-10
            assert abs(R[b]["finalcost"] - R0[b]["finalcost"]) <= 1e-12 * R0[b]["finalcost"]
    plan.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_tuned_plan_solves_like_default(gpulib, c0, precision):
    prec = gpulib.FP64 if precision == "fp64" else gpulib.FP32
    plan, probs = _plan(gpulib, c0, prec)
    X0, R0 = _solve(plan, probs)
    shapes, ms = plan.tune(reps=3)
    assert shapes == plan.shapes()
    assert 1 <= shapes["interp_ppw"] <= 16 and 1 <= shapes["spread_cluster"] <= 16
    assert shapes["rows_per_cta"] >= 1 and shapes["cols_per_cta"] >= 1
    assert all(v > 0 for v in ms.values())
    X, R = _solve(plan, probs)
    # FP64: rounding-level moves; FP32: regrouped FP32 sums move the
    # (unconverged) 150-iteration images by ~1e-4 and objectives by ~1e-6
    xtol, ftol = (1e-10, 1e-12) if precision == "fp64" else (2e-3, 1e-5)
    for b in range(len(probs)):
        assert rel(X[b], X0[b]) < xtol
        assert abs(R[b]["finalcost"] - R0[b]["finalcost"]) <= ftol * R0[b]["finalcost"]
    plan.close()


def test_impossible_shapes_are_rejected(gpulib, c0):
    plan, probs = _plan(gpulib, c0)
    before = plan.shapes()
    for bad in [dict(interp_ppw=64), dict(spread_cluster=32), dict(rows_per_cta=10000)]:
        with pytest.raises(gpulib.MfistaError):
            plan.set_shapes(**bad)
    assert plan.shapes() == before
    X, R = _solve(plan, probs)   # the plan still runs
    assert all(np.isfinite(r["finalcost"]) for r in R)
    plan.close()
