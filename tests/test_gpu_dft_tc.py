"""DFT operator on the tensor cores (split BF16, tcgen05) against FP64.

The GEMM alone (no anchor) carries ~2^-16 relative error per product; the
solver applies it only to departures from an FP64 anchor, so a BF16X3 batch
reaches the FP64 batch's objective.  Shapes cover padding of every operand
(rows to 128, K to 64, problems to 64).
"""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


def _rand(m, n, b, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((m, n)), rng.standard_normal((b, n)), rng.standard_normal((b, m))


@pytest.mark.parametrize("m,n,b", [(300, 256, 3), (1000, 900, 70), (2000, 1024, 64)])
def test_dft_apply_fp64_exact(gpulib, m, n, b):
    A, X, R = _rand(m, n, b, m + n)
    assert rel(gpulib.dft_apply(A, X), X @ A.T) < 1e-13
    assert rel(gpulib.dft_apply(A, R, transpose=True), R @ A) < 1e-13


@pytest.mark.parametrize("form,tol", [("bf16x3", 5e-5), ("bf16x6", 1e-5)])
@pytest.mark.parametrize("m,n,b", [(300, 256, 3), (1000, 900, 70), (2000, 1024, 64)])
def test_dft_apply_split_bf16_tensor_cores(gpulib, m, n, b, form, tol):
    """Three products of two-plane operands (~2^-16 per product), or six of
    three-plane operands (FP32 accumulation then dominates, ~1e-6)."""
    prec = gpulib.BF16X3 if form == "bf16x3" else gpulib.BF16X6
    A, X, R = _rand(m, n, b, m * n)
    ref_f, ref_a = X @ A.T, R @ A
    f = gpulib.dft_apply(A, X, precision=prec)
    a = gpulib.dft_apply(A, R, transpose=True, precision=prec)
    # per-row check too: every problem (including those past a 64-problem
    # tile boundary) and every padded row boundary
    assert rel(f, ref_f) < tol and rel(a, ref_a) < tol
    for k in range(b):
        assert rel(f[k], ref_f[k]) < 2 * tol and rel(a[k], ref_a[k]) < 2 * tol
    # deterministic: the same call gives the same bits
    assert np.array_equal(f, gpulib.dft_apply(A, X, precision=prec))


@pytest.mark.parametrize("form", ["bf16x3", "bf16x6"])
def test_dft_batch_split_bf16_reaches_fp64_objective(gpulib, form):
    """The split-BF16 batch reaches the FP64 batch's objective (after 800 FP64
    iterations) to 1e-6 relative, as the FP32 NUFFT form does.  Images that
    close in objective still differ by a few percent on this small,
    ill-conditioned problem (the optimum is flat), hence the looser image
    bound."""
    from sparseimaging_b200 import synth
    p = synth.dft_problem(nx=32, n_stations=8, n_hours=40, seed=5, m_vis=1000)
    A, y = p.A, p.y
    g0 = np.abs(A.T @ y).max()
    lip = np.linalg.norm(A, 2) ** 2
    probs = [dict(lambda_l1=g0 * s, lambda_tsv=g0 * s * 1e-2, cinit=lip, maxiter=800, nonneg_flag=1)
             for s in (3e-3, 1e-2, 3e-2, 1e-1)]
    X64, R64 = gpulib.dft_batch(y, A, 32, 32, probs, 0.0)
    targets = [r["finalcost"] * (1 + 1e-6) for r in R64]
    for q, t in zip(probs, targets):
        q["target_cost"] = t
        q["maxiter"] = 4000
    prec = gpulib.BF16X3 if form == "bf16x3" else gpulib.BF16X6
    X3, R3 = gpulib.dft_batch(y, A, 32, 32, probs, 0.0, precision=prec)
    for b, (r, t) in enumerate(zip(R3, targets)):
        assert r["finalcost"] <= t, (b, r["finalcost"], t)
        assert r["ITER"] < 4000
        assert rel(X3[b], X64[b]) < 1e-1
