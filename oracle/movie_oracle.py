"""CPU oracle of the movie solver (test infrastructure only).

TEST INFRASTRUCTURE ONLY: `tests/` use it as the checker; the library never
calls it.

Restates the reference's matlab/MFISTA_movie_eht.m (:93-194): the frames of
a movie are ONE problem,

  F(X) = sum_b [ chi2_b(x_b) / 2 + lam2 TSV(x_b) ] + lam_t dX(X),
  dX(X) = sum_b sum_i (x_b,i - x_{b+1},i)^2 / (t_{b+1} - t_b)   (matlab/lib/d_X.m)

with gradient terms dtX (matlab/lib/dt_X.m) and lam |X|_1, solved by MFISTA
with ONE step size c, momentum mu, backtracking test and stopping rule
(t > MINITER and cost(t - TD) - cost(t) < EPS, EPS unscaled; the matlab code
has no "x becomes a 0 vector" stop; its backtracking also ends once
c > 1e200).  The matlab code calls FINUFFT; here each frame uses the C
reference's NUFFT as restated in oracle/mfista_oracle.py (NufftPlan), as the
library does.  The matlab code cannot run here (no MATLAB/Octave), so this
restatement is pinned only through its single-frame, lam_t = 0 case, which
must equal the C reference's MFISTA loop (tests/test_movie_oracle.py).
"""
from __future__ import annotations

import math

import numpy as np

from .mfista_oracle import ETA, MINITER, TD, NufftPlan, d_tsv, nufft_f_part, nufft_grad, soft_threshold, \
    soft_threshold_nonneg, tsv


def d_x(X, wt):
    """sum_b wt_b |x_b - x_{b+1}|^2 (X is [T][N])."""
    if X.shape[0] < 2:
        return 0.0
    D = X[:-1] - X[1:]
    return float(np.sum(np.sum(D * D, axis=1) * wt))


def dt_x(X, wt):
    """Gradient of d_x."""
    G = np.zeros_like(X)
    if X.shape[0] < 2:
        return G
    tmp = 2 * (X[:-1] - X[1:]) * wt[:, None]
    G[:-1] += tmp
    G[1:] -= tmp
    return G


def movie(frames, nx, ny, lam, lam2, lam_t, cinit, maxiter, eps, nonneg_flag=1, t_list=None, xinit=None,
          c_box=None):
    """frames: list of (u, v, vis_r, vis_i, vis_std).  c_box: [N] pixel
    weights or None (x = xinit .* c_box, :46; every thresholded image times
    c_box, :143-146).  Returns (X [T][N], iterations, c, cost history)."""
    T = len(frames)
    N = nx * ny
    t = np.arange(1, T + 1, dtype=np.float64) if t_list is None else np.asarray(t_list, np.float64)
    wt = 1.0 / (t[1:] - t[:-1])
    ops = []
    for (u, v, vr, vi, vs) in frames:
        plan = NufftPlan(u, v, nx, ny)
        w = 1.0 / np.asarray(vs, np.float64)
        ops.append((plan, np.asarray(vr, np.float64), np.asarray(vi, np.float64), w))
    soft = soft_threshold_nonneg if nonneg_flag == 1 else soft_threshold
    box = None if c_box is None else np.asarray(c_box, np.float64)

    def prox(v, eta):
        out = soft(v, eta)
        return out if box is None else out * box[None, :]

    def frame_costs(X):
        """sum_b chi2_b/2 + lam2 TSV(x_b), and the residuals."""
        tot, res = 0.0, []
        for b, (plan, vr, vi, w) in enumerate(ops):
            f, r = nufft_f_part(plan, vr, vi, w, X[b])
            tot += f + (lam2 * tsv(nx, ny, X[b]) if lam2 > 0 else 0.0)
            res.append(r)
        return tot, res

    x0 = np.zeros(N) if xinit is None else np.asarray(xinit, np.float64)
    if box is not None:
        x0 = x0 * box
    X = np.tile(x0, (T, 1))
    Z = X.copy()
    c, mu = float(cinit), 1.0
    f0, _ = frame_costs(X)
    cost_now = f0 + lam * np.abs(X).sum()
    cost = np.zeros(maxiter)
    it = 0
    while it < maxiter:
        cost[it] = cost_now
        qcore, res = frame_costs(Z)
        qcore += lam_t * d_x(Z, wt)
        G = np.array([nufft_grad(ops[b][0], ops[b][3], res[b]) for b in range(T)])
        if lam2 > 0:
            G -= lam2 * np.array([d_tsv(nx, ny, Z[b]) for b in range(T)])
        G -= lam_t * dt_x(Z, wt)
        trial = 0
        while True:
            Xn = prox(G * (1.0 / c) + Z, lam / c)
            fval, _ = frame_costs(Xn)
            fval += lam_t * d_x(Xn, wt)
            D = Xn - Z
            qval = qcore + sum(-(G[b] @ D[b]) + c * (D[b] @ D[b]) / 2 for b in range(T))
            if fval <= qval:
                break
            c *= ETA
            trial += 1
            if trial >= maxiter or c > 1.0e200:
                break
        c /= ETA
        munew = (1 + math.sqrt(1 + 4 * mu * mu)) / 2
        fval += lam * np.abs(Xn).sum()
        if fval < cost[it]:
            cost_now = fval
            Z = X * ((1 - mu) / munew) + Xn * (1 + (mu - 1) / munew)
            X = Xn.copy()
        else:
            Z = X * (1 - mu / munew) + Xn * (mu / munew)
        if it >= MINITER and (cost[it - TD] - cost[it]) < eps:
            break
        mu = munew
        it += 1
    if it == maxiter:
        it -= 1
    return X, it + 1, c, cost[: it + 1]
