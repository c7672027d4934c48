"""A problem's result does not depend on the rest of its batch.

Shared-geometry launches cut the batch's ACTIVE problems into chunks anew
each time (a problem's chunk and slot change as others stop), and the FP32
interpolation takes a chunk's problems 8, 4, 2 or 1 at a time.  Every
kernel still forms each problem's sums in a fixed order of its own (the
grouped interpolation's transposing reduction adds the same lane pairs as a
plain butterfly), so a problem solved among others that stop at other
iterations gives the same bits as in a batch of its own.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problems(c0, scales, maxiters):
    lam1, lip = float(c0["lam1"]), float(c0["cinit"])
    return [dict(lambda_l1=lam1 * s, lambda_tsv=lam1 * 1e-3 * s, cinit=lip, maxiter=int(m), nonneg_flag=1)
            for s, m in zip(scales, maxiters)]


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_result_is_independent_of_batch_company(gpulib, c0, precision):
    prec = gpulib.FP32 if precision == "fp32" else gpulib.FP64
    geo = (c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"], 64, 64)
    mine = _problems(c0, np.geomspace(0.3, 3.0, 4), [300] * 4)
    # 17 others: other lambdas, stopping after 20..300 iterations, so the
    # active set (and every chunking of it) changes throughout the solve
    rng = np.random.default_rng(5)
    others = _problems(c0, rng.uniform(0.1, 10.0, 17), rng.integers(20, 300, 17))
    pos = [1, 6, 13, 20]
    batch, it = [], iter(others)
    for i in range(21):
        batch.append(mine[pos.index(i)] if i in pos else next(it))
    Xa, Ra = gpulib.nufft_batch(*geo, mine, 1e-6, precision=prec)
    Xb, Rb = gpulib.nufft_batch(*geo, batch, 1e-6, precision=prec)
    assert len({r["ITER"] for r in Rb}) > 4  # the company really stops at other times
    for j, i in enumerate(pos):
        assert Rb[i]["ITER"] == Ra[j]["ITER"]
        assert Rb[i]["finalcost"] == Ra[j]["finalcost"]
        assert np.array_equal(Xb[i], Xa[j])
