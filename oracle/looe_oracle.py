"""CPU oracle of the leave-one-out error (LOOE) of a DFT solution.

TEST INFRASTRUCTURE ONLY: `tests/` and `bench.py`'s CPU leg use this module
as the checker; the library never calls it.

The reference computes an approximate leave-one-out error of an L1 (or
L1 + TSV) solution from its active set (c/looe_lib.c; its call in
c/mfista_dft_lib.c:506-529 is commented out and the reference's makefile does
not build the file).  `looe` restates it in numpy:

* active set S = {j : |x_j| > 0} (find_active_set, :49-63);
* A_S = the columns of A in S (shrink_A, :67-81);
* H = A_S^T A_S (dsyrk, :181-204), plus lambda_tsv * d2(j) on the diagonal
  for the TSV form, d2 = 8 inside, 6 on an edge, 4 on a corner of the NX
  grid (d2_TSV, :228-245, column bound also taken from NX; compute_Hessian_
  L1_TSV, :247-273);
* d_i = (A_S H^-1 A_S^T)_ii (dposv on A_S^T, then the row dot products,
  compute_LOOE_core :112-171);
* t_i = (y - A x)_i / (1 - d_i), s_i = t_i^2 / 2;
  LOOE_m = mean(s), LOOE_std = sqrt(sum(s^2)/(M-1) - LOOE_m^2 M/(M-1));
* a Hessian that is not positive definite gives (-1, 0, 0): the reference
  returns -1 with both outputs left at 0.

`looe_ref` calls the reference's own compute_LOOE_L1 / compute_LOOE_L1_TSV,
compiled from the reference sources into oracle/_ref/liblooe_ref.so by
oracle/Makefile (with project-written dsyrk_/dposv_ loops in
oracle/shim/lapack_shim.c); it pins the restatement.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "liblooe_ref.so")


def d2_tsv(j, nx):
    """Diagonal of the TSV Hessian for pixel j (c/looe_lib.c:228-245)."""
    r = j % nx
    c = j // nx
    r_in = 0 < r < nx - 1
    c_in = 0 < c < nx - 1
    if r_in:
        return 8.0 if c_in else 6.0
    return 6.0 if c_in else 4.0


def looe(y, A, x, nx, lambda_tsv=0.0):
    """(status, looe_m, looe_std): status 1 = Hessian positive definite,
    0 = not (looe_m = looe_std = 0).  A is (M, N); x has N entries."""
    y = np.asarray(y, np.float64)
    A = np.asarray(A, np.float64)
    x = np.asarray(x, np.float64)
    M = A.shape[0]
    S = np.flatnonzero(np.abs(x) > 0)
    As = A[:, S]
    H = As.T @ As
    if lambda_tsv != 0.0:
        H[np.diag_indices_from(H)] += lambda_tsv * np.array([d2_tsv(int(j), nx) for j in S])
    try:
        L = np.linalg.cholesky(H)
    except np.linalg.LinAlgError:
        return 0, 0.0, 0.0
    Z = np.linalg.solve(L, As.T)          # L^-1 A_S^T
    d = np.sum(Z * Z, axis=0)             # (A_S H^-1 A_S^T)_ii
    r = y - A @ x
    t = r / (1.0 - d)
    s = t * t / 2
    m = float(np.mean(s))
    var = float(np.sum(s * s) / (M - 1) - m * m * M / (M - 1))
    return 1, m, float(np.sqrt(var))


def looe_ref(y, A, x, nx, ny, lambda_l1, lambda_tsv=0.0):
    """The reference's own LOOE (compiled c/looe_lib.c): (status, m, std)."""
    L = C.CDLL(REF_LIB)
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    y = np.ascontiguousarray(y, np.float64)
    A = np.asarray(A, np.float64)
    Af = np.asfortranarray(A)
    x = np.ascontiguousarray(x, np.float64)
    M, N = A.shape
    yAx = np.ascontiguousarray(y - A @ x)
    m, n = C.c_int(M), C.c_int(N)
    om, os_ = C.c_double(0), C.c_double(0)
    P = lambda a: a.ctypes.data_as(dp)
    if lambda_tsv == 0.0:
        L.compute_LOOE_L1.restype = C.c_double
        L.compute_LOOE_L1.argtypes = [ip, ip, C.c_double, dp, dp, dp, dp, dp, dp]
        v = L.compute_LOOE_L1(C.byref(m), C.byref(n), lambda_l1, P(y), Af.ctypes.data_as(dp), P(x), P(yAx),
                              C.byref(om), C.byref(os_))
    else:
        L.compute_LOOE_L1_TSV.restype = C.c_double
        L.compute_LOOE_L1_TSV.argtypes = [ip, ip, C.c_int, C.c_int, C.c_double, C.c_double, dp, dp, dp, dp, dp, dp]
        v = L.compute_LOOE_L1_TSV(C.byref(m), C.byref(n), nx, ny, lambda_l1, lambda_tsv, P(y),
                                  Af.ctypes.data_as(dp), P(x), P(yAx), C.byref(om), C.byref(os_))
    if v == -1.0:
        return 0, float(om.value), float(os_.value)
    return 1, float(om.value), float(os_.value)
