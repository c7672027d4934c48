"""Leave-one-out error on the GPU (mfista_dft_looe) against the oracle.

The reference's own c/looe_lib.c pins the numpy restatement
(tests/test_looe_oracle.py); here the GPU's FP64 blocked Cholesky and
triangular solve (other summation orders than the reference's dposv) must
agree with it to 1e-9 relative on well-posed Hessians, report the same
not-positive-definite case, and give the same bits on a repeated call."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..")
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
from oracle import looe_oracle as O  # noqa: E402
import make_looe_golden as G  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _close(a, b, tol=TOL):
    return abs(a - b) <= tol * abs(b)


def test_looe_matches_reference_fixture(gpulib):
    d = np.load(os.path.join(ROOT, "tests", "golden", "looe_small.npz"))
    y, A, x, nx = d["y"], d["A"], d["x"], int(d["nx"])
    for name, (Ac, xc, lt) in G.cases(y, A, x).items():
        want = d[f"{name}_out"]
        m, sd, pos = gpulib.dft_looe(y, Ac, xc[None], nx, lambda_tsv=[lt])
        assert bool(pos[0]) == bool(want[0]), name
        if want[0]:
            assert _close(m[0], want[1]) and _close(sd[0], want[2]), (name, m[0], want[1])
        else:
            assert m[0] == 0.0 and sd[0] == 0.0


@pytest.mark.parametrize("lt", [0.0, 0.5])
def test_looe_blocked_sizes(gpulib, lt):
    """Active sets of 1 to ~330 pixels: one and several 64-wide Cholesky
    panels, ragged last panels, GEMM edge tiles; M = 2000 rows."""
    rng = np.random.default_rng(7)
    nx = 32
    M, N = 2000, nx * nx
    A = rng.normal(size=(M, N)) / np.sqrt(M)
    X = []
    for frac in (0.001, 0.06, 0.13, 0.32):
        x = np.where(rng.random(N) < frac, rng.random(N), 0.0)
        if not x.any():
            x[5] = 1.0
        X.append(x)
    X = np.array(X)
    y = A @ X[2] + 0.01 * rng.normal(size=M)
    m, sd, pos = gpulib.dft_looe(y, A, X, nx, lambda_tsv=lt)
    for b in range(len(X)):
        st, wm, wsd = O.looe(y, A, X[b], nx, lt)
        assert st == 1 and pos[b]
        assert _close(m[b], wm) and _close(sd[b], wsd), (b, m[b], wm, sd[b], wsd)
    m2, sd2, pos2 = gpulib.dft_looe(y, A, X, nx, lambda_tsv=lt)
    assert np.array_equal(m, m2) and np.array_equal(sd, sd2) and np.array_equal(pos, pos2)


def test_looe_of_dft_lambda_grid_solutions(gpulib):
    """LOOE of solutions from the batched DFT solver (the use the reference
    wrote it for: choosing lambda), L1 + TSV form."""
    from sparseimaging_b200 import synth
    p = synth.dft_problem(nx=32, n_stations=8, n_hours=40, seed=5, m_vis=1000)
    A, y = p.A, p.y
    g0 = np.abs(A.T @ y).max()
    lip = np.linalg.norm(A, 2) ** 2
    scales = (3e-3, 1e-2, 3e-2, 1e-1)
    probs = [dict(lambda_l1=g0 * s, lambda_tsv=g0 * s * 1e-2, cinit=lip, maxiter=500, nonneg_flag=1)
             for s in scales]
    X, _ = gpulib.dft_batch(y, A, 32, 32, probs, 0.0)
    lts = [q["lambda_tsv"] for q in probs]
    m, sd, pos = gpulib.dft_looe(y, A, X, 32, lambda_tsv=lts)
    for b in range(len(probs)):
        st, wm, wsd = O.looe(y, A, X[b], 32, lts[b])
        assert bool(pos[b]) == bool(st)
        if st:
            assert _close(m[b], wm, 1e-8) and _close(sd[b], wsd, 1e-8), (b, m[b], wm)


def test_looe_rejects_bad_arguments(gpulib):
    A = np.ones((1, 4))
    with pytest.raises(gpulib.MfistaError):
        gpulib.dft_looe(np.ones(1), A, np.ones((1, 4)), 2)
