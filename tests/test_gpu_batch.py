"""Batched solves: per-problem state and masks on the device.

Every problem of an FP64 batch must reproduce the single-problem drop-in
solve with the same parameters (the kernels never mix problems, so the
arithmetic is identical); the FP32 form is checked against FP64.
"""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


def _single(si, c0, lam1, lts, maxiter, nonneg=1):
    return si.imaging_core_nufft(c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"], 64, 64,
                                 maxiter, 1e-5, lam1, 0.0, lts, float(c0["cinit"]), nonneg_flag=nonneg)


def _problems(c0, scales, maxiter):
    lam1 = float(c0["lam1"])
    return [dict(lambda_l1=lam1 * s, lambda_tsv=lam1 * 1e-3 * s, cinit=float(c0["cinit"]),
                 maxiter=maxiter, nonneg_flag=1) for s in scales]


def test_shared_geometry_batch_equals_single_solves(gpulib, c0):
    scales = [0.3, 1.0, 4.0]
    probs = _problems(c0, scales, 120)
    X, R = gpulib.nufft_batch(c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"], 64, 64,
                              probs, 1e-5)
    for b, p in enumerate(probs):
        x, r = _single(gpulib, c0, p["lambda_l1"], p["lambda_tsv"], 120)
        assert R[b]["ITER"] == r["ITER"]
        assert rel(X[b], x) < 1e-13
        assert abs(R[b]["finalcost"] - r["finalcost"]) <= 1e-13 * r["finalcost"]


def test_uneven_geometry_batch_equals_single_solves(gpulib, c0):
    """Three problems with 2016, 1200 and 700 points in one launch."""
    m = c0["u"].size
    sizes = [m, 1200, 700]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    cat = lambda a: np.concatenate([a[:s] for s in sizes])
    probs = _problems(c0, [1.0, 1.0, 1.0], 100)
    X, R = gpulib.nufft_batch(cat(c0["u"]), cat(c0["v"]), cat(c0["vis_r"]), cat(c0["vis_i"]),
                              cat(c0["vis_std"]), 64, 64, probs, 1e-5, pt_off=off)
    for b, s in enumerate(sizes):
        x, r = gpulib.imaging_core_nufft(c0["u"][:s], c0["v"][:s], c0["vis_r"][:s], c0["vis_i"][:s],
                                         c0["vis_std"][:s], 64, 64, 100, 1e-5, probs[b]["lambda_l1"], 0.0,
                                         probs[b]["lambda_tsv"], probs[b]["cinit"])
        assert R[b]["ITER"] == r["ITER"] and R[b]["M"] == s // 2
        assert rel(X[b], x) < 1e-13


def test_fp32_form_against_fp64(gpulib, c0):
    """FP32 operators: the objective tracks FP64 to the FP32 floor (~1e-5
    relative on this data: 1 % noise under the model values)."""
    probs = _problems(c0, [0.5, 1.0, 2.0, 8.0], 150)
    args = (c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"], 64, 64, probs, 1e-5)
    X64, R64 = gpulib.nufft_batch(*args)
    X32, R32 = gpulib.nufft_batch(*args, precision=gpulib.FP32)
    for b in range(len(probs)):
        assert rel(X32[b], X64[b]) < 1e-2
        assert abs(R32[b]["finalcost"] - R64[b]["finalcost"]) <= 5e-5 * R64[b]["finalcost"]


def test_plan_reuse_is_deterministic(gpulib, c0):
    probs = _problems(c0, [0.7, 1.3], 80)
    plan = gpulib.Plan(c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"], 64, 64, 2)
    plan.set_problems(probs, 1e-5)
    plan.run()
    X1, R1 = plan.fetch()
    plan.set_problems(probs, 1e-5)
    plan.run()
    X2, R2 = plan.fetch()
    assert np.array_equal(X1, X2)
    assert [r["ITER"] for r in R1] == [r["ITER"] for r in R2]
    assert plan.kernel_launches > 80
    assert plan.device_loop, "conditional WHILE graph node not in use"
    plan.close()


def test_tv_batch_equals_single(gpulib, c0):
    lam1 = float(c0["lam1"])
    probs = [dict(lambda_l1=lam1, lambda_tv=5e-3 * lam1 * s, cinit=float(c0["cinit"]), maxiter=30,
                  nonneg_flag=1) for s in (1.0, 3.0)]
    X, R = gpulib.nufft_batch(c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"], 64, 64, probs,
                              1e-5)
    for b, p in enumerate(probs):
        x, r = gpulib.imaging_core_nufft(c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"], 64, 64,
                                         30, 1e-5, lam1, p["lambda_tv"], 0.0, p["cinit"])
        assert R[b]["ITER"] == r["ITER"]
        assert rel(X[b], x) < 1e-13


def test_nan_visibility_stops_with_status(gpulib, c0):
    """NaN data never passes the backtracking test; the problem stops with
    MFISTA_ERR_NONFINITE (5) instead of retrying maxiter times per iteration."""
    vr = c0["vis_r"].copy()
    vr[3] = np.nan
    probs = _problems(c0, [1.0], 1000)
    with pytest.raises(gpulib.MfistaError) as e:
        gpulib.nufft_batch(c0["u"], c0["v"], vr, c0["vis_i"], c0["vis_std"], 64, 64, probs, 1e-5)
    assert e.value.status == 5


def test_batch_rejects_mixed_regularisers(gpulib, c0):
    probs = _problems(c0, [1.0], 10)
    probs[0]["lambda_tv"] = 1.0
    with pytest.raises(gpulib.MfistaError):
        gpulib.nufft_batch(c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"], 64, 64, probs, 1e-5)


def test_fp32_defect_corrected_reaches_fp64_objective(gpulib, c0):
    """FP32 operators with the FP64 anchor correction reach the FP64
    objective to 1e-6 relative (the uncorrected FP32 form stalls near 1e-5)."""
    probs = _problems(c0, [0.5, 2.0], 1200)
    geo = (c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"], 64, 64)
    X64, R64 = gpulib.nufft_batch(*geo, probs, 0.0)
    targets = [r["finalcost"] * (1 + 1e-6) for r in R64]
    for p, t in zip(probs, targets):
        p["target_cost"] = t
        p["maxiter"] = 4000
    X32, R32 = gpulib.nufft_batch(*geo, probs, 0.0, precision=gpulib.FP32)
    for b, (r, t) in enumerate(zip(R32, targets)):
        assert r["finalcost"] <= t, (b, r["finalcost"], t)
        assert r["ITER"] < 4000
        assert rel(X32[b], X64[b]) < 2e-2


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_device_loop_matches_host_loop(gpulib, c0, precision, monkeypatch):
    """The device loop (CUDA graph WHILE node whose anchor-refresh and
    gradient blocks sit under IF nodes, skipped in steps that need neither)
    gives the host loop's bits (every kernel launched each step, gated per
    problem).  With anchor refreshes every 32 iterations (FP32 form) it
    launches fewer kernels; FP64 has no refresh block, and its gradient
    block is skipped only in backtracking retries."""
    prec = gpulib.FP32 if precision == "fp32" else gpulib.FP64
    probs = _problems(c0, [0.4, 1.0, 3.0], 120)
    args = (c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"], 64, 64, len(probs))
    out = {}
    for mode in ("device", "host"):
        if mode == "host":
            monkeypatch.setenv("MFISTA_HOST_LOOP", "1")
        plan = gpulib.Plan(*args, precision=prec)
        plan.set_problems(probs, 1e-5)
        plan.run()
        X, R = plan.fetch()
        out[mode] = (X, R, plan.kernel_launches, plan.device_loop)
        plan.close()
    (Xd, Rd, Ld, dd), (Xh, Rh, Lh, dh) = out["device"], out["host"]
    assert dd and not dh
    assert np.array_equal(Xd, Xh)
    assert [r["ITER"] for r in Rd] == [r["ITER"] for r in Rh]
    assert [r["finalcost"] for r in Rd] == [r["finalcost"] for r in Rh]
    if precision == "fp32":
        assert Ld < Lh


def test_batch_rejects_offsets_beyond_the_arrays(gpulib, c0):
    """Independent geometry: pt_off[B] larger than M (the length of the
    concatenated point arrays) is rejected before anything reads them."""
    import ctypes as C
    m = 100
    u = np.ascontiguousarray(c0["u"][:m])
    arrs = [np.ascontiguousarray(c0[k][:m], np.float64) for k in ("u", "v", "vis_r", "vis_i", "vis_std")]
    off = np.array([0, 50, 150], np.int32)
    probs = gpulib._problems(_problems(c0, [1.0, 1.0], 10))
    xo = np.zeros(2 * 64 * 64)
    res = (gpulib.RESULT * 2)()
    dp = C.POINTER(C.c_double)
    st = gpulib.lib().mfista_nufft_batch(*[a.ctypes.data_as(dp) for a in arrs], off.ctypes.data_as(C.POINTER(C.c_int)),
                                         0, m, 64, 64, 2, probs, 1e-5, gpulib.FP64, 100, None,
                                         xo.ctypes.data_as(dp), res)
    assert st == 2
    assert u.size == m
