"""The drop-in NUFFT entry's solver cache (mfista_imaging_core_nufft).

A call with the same uv points, vis_std, sizes, form and box as an earlier
one reuses that call's solver and only uploads the new visibilities.  The
results must be the bits of a solver built afresh: new visibilities and
parameters on a kept geometry, a changed geometry (a miss), the TV form and
a box mask, and the cache switched off by the environment."""
import os
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("ITER", "finalcost", "sq_error", "l1cost", "tsvcost", "tvcost", "N_active", "Lip_const")


def _solve(si, c0, vis_r, vis_i, u=None, lam1=None, ltv=0.0, lts=None, box=None, maxiter=150):
    lam1 = float(c0["lam1"]) if lam1 is None else lam1
    lts = float(c0["lamt"]) if lts is None else lts
    t = time.perf_counter()
    x, r = si.imaging_core_nufft(c0["u"] if u is None else u, c0["v"], vis_r, vis_i, c0["vis_std"], 64, 64, maxiter,
                                 1e-5, lam1, ltv, lts, float(c0["cinit"]), box_flag=0 if box is None else 1,
                                 cl_box=box)
    return x, r, time.perf_counter() - t


def _fresh(si, *a, **k):
    si.release_cache()
    old = os.environ.get("MFISTA_DROPIN_CACHE")
    os.environ["MFISTA_DROPIN_CACHE"] = "0"
    try:
        return _solve(si, *a, **k)
    finally:
        if old is None:
            del os.environ["MFISTA_DROPIN_CACHE"]
        else:
            os.environ["MFISTA_DROPIN_CACHE"] = old


def _same(a, b):
    assert np.array_equal(a[0], b[0])
    for k in KEYS:
        assert a[1][k] == b[1][k], k


def test_cached_solver_gives_fresh_bits(gpulib):
    si = gpulib
    from conftest import load_golden
    c0 = load_golden("c0_nufft.npz")
    rng = np.random.default_rng(21)
    vr2 = c0["vis_r"] * 0.8 + 0.01 * rng.standard_normal(c0["vis_r"].size)
    vi2 = c0["vis_i"] * 0.8 + 0.01 * rng.standard_normal(c0["vis_i"].size)
    si.release_cache()
    first = _solve(si, c0, c0["vis_r"], c0["vis_i"])                       # miss: builds and keeps
    hit = _solve(si, c0, vr2, vi2, lam1=0.5 * float(c0["lam1"]))            # hit: new data and lambda
    ref = _fresh(si, c0, vr2, vi2, lam1=0.5 * float(c0["lam1"]))
    _same(hit, ref)
    again = _solve(si, c0, c0["vis_r"], c0["vis_i"])                       # the first call's data again
    _same(again, first)
    u2 = c0["u"].copy()
    u2[0] += 1e-9                                                            # another geometry: a miss
    _same(_solve(si, c0, vr2, vi2, u=u2), _fresh(si, c0, vr2, vi2, u=u2))
    # setup skipped: the call's time outside the solve
    assert hit[2] - hit[1]["comp_time"] < first[2] - first[1]["comp_time"]


def test_cache_keys_form_and_box(gpulib):
    si = gpulib
    from conftest import load_golden
    c0 = load_golden("c0_nufft.npz")
    si.release_cache()
    lam_tv = float(c0["lamt"])
    tv = _solve(si, c0, c0["vis_r"], c0["vis_i"], ltv=lam_tv, lts=0.0, maxiter=60)
    tsv = _solve(si, c0, c0["vis_r"], c0["vis_i"], maxiter=60)
    _same(tv, _fresh(si, c0, c0["vis_r"], c0["vis_i"], ltv=lam_tv, lts=0.0, maxiter=60))
    _same(tsv, _fresh(si, c0, c0["vis_r"], c0["vis_i"], maxiter=60))
    box = np.zeros(64 * 64, np.float32)
    box.reshape(64, 64)[16:48, 16:48] = 1
    b1 = _solve(si, c0, c0["vis_r"], c0["vis_i"], box=box, maxiter=60)
    b2 = _solve(si, c0, c0["vis_r"], c0["vis_i"], box=box, maxiter=60)
    _same(b1, b2)
    _same(b1, _fresh(si, c0, c0["vis_r"], c0["vis_i"], box=box, maxiter=60))
    assert np.all(b1[0].reshape(64, 64)[:16] == 0)
    si.release_cache()
