"""CPU restatement (numpy, FP64) of the sparseimaging MFISTA solver path.

TEST INFRASTRUCTURE ONLY.  This module is the parity checker: tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may call it, nothing in
the shipped library does.  It restates, in vectorised numpy, what the reference
C solvers compute; every function cites the reference lines it follows.  It is
pinned against the reference itself, compiled unchanged by oracle/Makefile into
oracle/_ref/ (see tests/test_oracle.py and tests/golden/make_golden.py).

Array layouts are the reference's: images are flat ``x[i*Ny + j]`` for the
NUFFT variant; TSV/TV/FGP view the same flat array as NY rows of NX
(``x[NX*j + i]``, c/mfista_tools.c:145-186, c/mfista_TV_lib.c:30-122).
"""
from __future__ import annotations

import math
import numpy as np

# c/mfista.h:36-41 and c/mfista_nufft_lib.c:27-28
MAXITER = 50000
MINITER = 100
FGPITER = 100
TD = 50
ETA = 1.1
EPS = 1.0e-5
MSP = 12
NU_SIGN = -1
TAPS = 2 * MSP


# --------------------------------------------------------------------------
# index helpers (c/mfista_nufft_lib.c:32-48)
# --------------------------------------------------------------------------

def wrap_index(m, mr):
    """idx_fftw (c/mfista_nufft_lib.c:32-40): m in [-mr/2, mr/2) -> m mod mr.
    Anything else lands outside the reference's array; -1 here (dropped)."""
    m = np.asarray(m)
    h = mr // 2
    return np.where((m >= -h) & (m < h), np.mod(m, mr), -1)


def half_col(m, ny):
    """Column of the half-plane grid (ny+1 columns) that the reference accepts
    for y index m (c/mfista_nufft_lib.c:154-156,218): idx_fftw(m, 2ny) < ny+1,
    i.e. m in [0, ny) -> m and m == -ny -> ny; -1 otherwise."""
    c = wrap_index(m, 2 * ny)
    return np.where((c >= 0) & (c < ny + 1), c, -1)


def centre_index(idx, n):
    """m2mr (c/mfista_nufft_lib.c:42-48)."""
    idx = np.asarray(idx)
    return np.where(idx < n // 2, idx + (3 * n) // 2, idx - n // 2)


# --------------------------------------------------------------------------
# NUFFT (c/mfista_nufft_lib.c:50-304)
# --------------------------------------------------------------------------

class NufftPlan:
    """Grid-correction factors and tap geometry of preNUFFT
    (c/mfista_nufft_lib.c:50-121), plus vectorised gather/scatter indices."""

    def __init__(self, u, v, nx, ny):
        u = np.asarray(u, np.float64)
        v = np.asarray(v, np.float64)
        self.nx, self.ny, self.m = nx, ny, u.size
        mrx, mry = 2.0 * nx, 2.0 * ny
        taux = 12.0 / float(nx * nx)
        tauy = 12.0 / float(ny * ny)
        coeff = math.pi / math.sqrt(taux * tauy)
        l = np.arange(MSP + 1, dtype=np.float64)
        self.e3x = np.exp(-((math.pi / mrx) ** 2 / taux) * l * l)
        self.e3y = np.exp(-((math.pi / mry) ** 2 / tauy) * l * l)
        # note the reference centres both axes on Nx/2 here (:78, :82)
        ti = (np.arange(nx) - nx // 2).astype(np.float64)
        tj = (np.arange(ny) - nx // 2).astype(np.float64)
        self.e4 = coeff * np.exp(taux * ti[:, None] ** 2 + tauy * tj[None, :] ** 2)
        tx = np.round(u * mrx / (2 * math.pi))
        ty = np.round(v * mry / (2 * math.pi))
        self.mx = tx.astype(np.int64)
        self.my = ty.astype(np.int64)
        dx = u - 2 * math.pi * tx / mrx
        dy = v - 2 * math.pi * ty / mry
        self.e1 = np.exp(-dx * dx / (4 * taux) - dy * dy / (4 * tauy))
        powj = np.arange(-MSP + 1, MSP + 1, dtype=np.float64)
        self.e2x = np.exp(powj[None, :] * (math.pi * dx / (mrx * taux))[:, None])
        self.e2y = np.exp(powj[None, :] * (math.pi * dy / (mry * tauy))[:, None])
        off = np.arange(-MSP + 1, MSP + 1)
        ab = np.abs(off)
        self.wx = self.e2x * self.e3x[ab][None, :]          # [M, 24]
        self.wy = self.e2y * self.e3y[ab][None, :]          # [M, 24]
        # tap cells: direct (m + l) and Hermitian mirror (-(m + l))
        gx = self.mx[:, None] + off[None, :]
        gy = self.my[:, None] + off[None, :]
        self.rx_d = wrap_index(gx, 2 * nx)
        self.rx_m = wrap_index(-gx, 2 * nx)
        self.cy_d = half_col(gy, ny)
        self.cy_m = half_col(-gy, ny)
        self.mm = float(2 * nx) * float(2 * ny)

    # -- padded image <-> half-plane grid --------------------------------
    def pad(self, x):
        """x*E4 into the centred 2Nx x 2Ny real grid (:202-208)."""
        nx, ny = self.nx, self.ny
        p = np.zeros((2 * nx, 2 * ny))
        ri = centre_index(np.arange(nx), nx)
        cj = centre_index(np.arange(ny), ny)
        p[np.ix_(ri, cj)] = np.asarray(x).reshape(nx, ny) * self.e4
        return p

    def unpad(self, p):
        """out[m2mr(k), m2mr(j)] * E4 / MM (:175-183), as a flat image."""
        nx, ny = self.nx, self.ny
        ri = centre_index(np.arange(nx), nx)
        cj = centre_index(np.arange(ny), ny)
        return (p[np.ix_(ri, cj)] * self.e4 / self.mm).reshape(-1)

    # -- forward: NUFFT2d2 (:187-243) -------------------------------------
    def _gather_tables(self):
        """Flat half-grid cells and weights of every (point, ly, lx) tap: the
        direct cells when the y index lands in the half plane, else the
        mirrored cell with the opposite sign on the imaginary part."""
        if getattr(self, "_fwd", None) is None:
            ny1 = self.ny + 1
            direct = self.cy_d >= 0
            col = np.where(direct, self.cy_d, self.cy_m)
            sgn = np.where(direct, NU_SIGN, -NU_SIGN).astype(np.float64)
            row = np.where(direct[:, :, None], self.rx_d[:, None, :], self.rx_m[:, None, :])
            ok = (col[:, :, None] >= 0) & (row >= 0)
            flat = np.where(ok, row * ny1 + col[:, :, None], 0).reshape(self.m, -1)
            w = ((self.e1[:, None, None] * self.wy[:, :, None]) * self.wx[:, None, :] / self.mm) * ok
            self._fwd = (flat, w.reshape(self.m, -1), (w * sgn[:, :, None]).reshape(self.m, -1))
        return self._fwd

    def forward(self, x):
        g = np.fft.rfft2(self.pad(x)).reshape(-1)   # FFTW r2c == rfft2 (unnormalised)
        flat, wr, wi = self._gather_tables()
        vals = g[flat]
        return np.einsum("kt,kt->k", wr, vals.real), np.einsum("kt,kt->k", wi, vals.imag)

    # -- adjoint: NUFFT2d1 (:123-185) -------------------------------------
    def _scatter_tables(self):
        if getattr(self, "_adj", None) is None:
            ny1 = self.ny + 1
            ww = (self.wy[:, :, None] * self.wx[:, None, :]) / 2          # [M, ly, lx]
            parts = []
            for rows, cols, conj in ((self.rx_d, self.cy_d, False), (self.rx_m, self.cy_m, True)):
                ok = (cols[:, :, None] >= 0) & (rows[:, None, :] >= 0)
                flat = (rows[:, None, :] * ny1 + cols[:, :, None])[ok]
                kidx = np.broadcast_to(np.arange(self.m)[:, None, None], ok.shape)[ok]
                parts.append((flat, kidx, ww[ok], conj))
            self._adj = parts
        return self._adj

    def adjoint(self, fin_r, fin_i):
        nx, ny = self.nx, self.ny
        size = 2 * nx * (ny + 1)
        v0 = np.asarray(fin_r) * self.e1 + 1j * (NU_SIGN * np.asarray(fin_i) * self.e1)
        acc = np.zeros(size, np.complex128)
        for flat, kidx, w, conj in self._scatter_tables():
            v = v0[kidx] * w
            if conj:
                v = np.conj(v)
            acc += np.bincount(flat, weights=v.real, minlength=size)
            acc += 1j * np.bincount(flat, weights=v.imag, minlength=size)
        g = acc.reshape(2 * nx, ny + 1)
        # FFTW c2r (unnormalised); numpy's irfft2 divides by the size
        p = np.fft.irfft2(g, s=(2 * nx, 2 * ny)) * self.mm
        return self.unpad(p)


def nufft_f_part(plan, vis_r, vis_i, weight, x):
    """calc_F_part_nufft (:258-285): residual (vis - A x) * w and chi^2/2."""
    fr, fi = plan.forward(x)
    rr = (vis_r - fr) * weight
    ri = (vis_i - fi) * weight
    return 0.5 * (rr @ rr + ri @ ri), (rr, ri)


def nufft_grad(plan, weight, resid):
    """dF_dx_nufft (:287-304): A^H of the residual weighted once more."""
    rr, ri = resid
    return plan.adjoint(rr * weight, ri * weight)


# --------------------------------------------------------------------------
# FFT variant (c/mfista_fft_lib.c:27-175)
# --------------------------------------------------------------------------

class FftOperator:
    """Gridded visibilities: mask and data on the half spectrum
    (idx2mat :70-88 then full2half/fft_full2half :50-68)."""

    def __init__(self, u_idx, v_idx, y_r, y_i, noise, nx, ny):
        self.nx, self.ny = nx, ny
        mk = np.zeros((nx, ny))
        yf = np.zeros((nx, ny), np.complex128)
        u_idx = np.asarray(u_idx)
        v_idx = np.asarray(v_idx)
        # sequential assignment semantics: last write wins on duplicates
        mk[u_idx, v_idx] = 1.0 / np.asarray(noise)
        yf[u_idx, v_idx] = (np.asarray(y_r) + 1j * np.asarray(y_i)) / np.asarray(noise)
        nyh = ny // 2 + 1
        self.mask_h = mk[:, :nyh].copy()
        self.yf_h = yf[:, :nyh].copy()
        # multiplicity of each half-spectrum column in the full plane
        # (fft_half2full :27-48 mirrors columns 1 .. NY_h-2)
        self.colw = np.ones(nyh)
        self.colw[1:nyh - 1] = 2.0
        self.sqrtn = math.sqrt(float(nx * ny))

    def f_part(self, x):
        """calc_F_part_fft (:142-159): |full-plane residual|^2 / 4."""
        xh = np.fft.rfft2(np.asarray(x).reshape(self.nx, self.ny))
        r = self.yf_h - self.mask_h * xh / self.sqrtn
        val = np.sum((r.real ** 2 + r.imag ** 2) * self.colw[None, :])
        return val / 4.0, r

    def grad(self, r):
        """dF_dx_fft (:161-175): c2r of r * mask / (2 sqrt N)."""
        g = r * (self.mask_h / (2 * self.sqrtn))
        return (np.fft.irfft2(g, s=(self.nx, self.ny)) * (self.nx * self.ny)).reshape(-1)


# --------------------------------------------------------------------------
# DFT variant (c/mfista_dft_lib.c:30-66, :253-278)
# --------------------------------------------------------------------------

class DftOperator:
    def __init__(self, y, A):
        self.y = np.asarray(y, np.float64)
        self.A = np.asarray(A, np.float64)   # (M, N) logical, any memory order

    def f_part(self, x):
        r = self.y - self.A @ x
        return 0.5 * (r @ r), r

    def grad(self, r):
        return self.A.T @ r


# --------------------------------------------------------------------------
# regularisers and proximal maps (c/mfista_tools.c, c/mfista_TV_lib.c)
# --------------------------------------------------------------------------

def _grid(x, nx, ny):
    return np.asarray(x).reshape(ny, nx)       # F[j, i] == x[NX*j + i]


def tsv(nx, ny, x):
    """TSV (c/mfista_tools.c:145-163): squared neighbour differences."""
    f = _grid(x, nx, ny)
    return float(np.sum((f[:, :-1] - f[:, 1:]) ** 2) + np.sum((f[:-1, :] - f[1:, :]) ** 2))


def d_tsv(nx, ny, x):
    """d_TSV (c/mfista_tools.c:165-186)."""
    f = _grid(x, nx, ny)
    d = np.zeros_like(f)
    d[:, :-1] += 2 * (f[:, :-1] - f[:, 1:])
    d[:, 1:] += 2 * (f[:, 1:] - f[:, :-1])
    d[:-1, :] += 2 * (f[:-1, :] - f[1:, :])
    d[1:, :] += 2 * (f[1:, :] - f[:-1, :])
    return d.reshape(-1)


def tv(nx, ny, x):
    """Isotropic TV with abs terms on the last row/column (c/mfista_TV_lib.c:30-46)."""
    f = _grid(x, nx, ny)
    a = f[:-1, :-1] - f[:-1, 1:]
    b = f[:-1, :-1] - f[1:, :-1]
    s = np.sum(np.sqrt(a * a + b * b))
    s += np.sum(np.abs(f[-1, :-1] - f[-1, 1:]))
    s += np.sum(np.abs(f[:-1, -1] - f[1:, -1]))
    return float(s)


def soft_threshold(v, eta, box=None):
    """soft_threshold / soft_threshold_box (c/mfista_tools.c:81-112)."""
    out = np.where(v >= eta, v - eta, np.where(v <= -eta, v + eta, 0.0))
    if box is not None:
        out = np.where(box == 0, 0.0, out)
    return out


def soft_threshold_nonneg(v, eta, box=None):
    """soft_threshold_nonneg(_box) (c/mfista_tools.c:114-141)."""
    out = np.where(v < eta, 0.0, v - eta)
    if box is not None:
        out = np.where(box == 0, 0.0, out)
    return out


def positive(v, box=None):
    """P_positive(_box) (c/mfista_TV_lib.c:77-93)."""
    out = np.where(v < 0, 0.0, v)
    if box is not None:
        out = np.where(box == 0, 0.0, out)
    return out


def lx(nx, ny, x):
    """Lx (c/mfista_TV_lib.c:48-57): forward differences, p:(NY,NX-1), q:(NY-1,NX)."""
    f = _grid(x, nx, ny)
    return f[:, :-1] - f[:, 1:], f[:-1, :] - f[1:, :]


def lpq(nx, ny, p, q):
    """Lpq (c/mfista_TV_lib.c:59-75): adjoint of Lx."""
    f = np.zeros((ny, nx))
    f[:, :-1] += p
    f[:, 1:] -= p
    f[:-1, :] += q
    f[1:, :] -= q
    return f.reshape(-1)


def p_pqiso(p, q):
    """Isotropic projection (c/mfista_TV_lib.c:95-122)."""
    r = np.empty_like(p)
    s = np.empty_like(q)
    t = np.maximum(1.0, np.sqrt(p[:-1, :] ** 2 + q[:, :-1] ** 2))
    r[:-1, :] = p[:-1, :] / t
    s[:, :-1] = q[:, :-1] / t
    t_row = np.maximum(1.0, np.abs(p[-1, :]))
    r[-1, :] = p[-1, :] / t_row
    t_col = np.maximum(1.0, np.abs(q[:, -1]))
    s[:, -1] = q[:, -1] / t_col
    return r, s


def fgp(nx, ny, b, lam_l1, lam_tv, iters, nonneg, box=None):
    """FGP_L1(_box) / FGP_nonneg(_box) (c/mfista_TV_lib.c:124-384).

    nonneg=True uses the P_positive projection (lam_l1 is ignored, the caller
    folds -lam_l1/c into b as c/mfista_nufft_lib.c:424-434 does)."""
    b = np.asarray(b)
    p = np.zeros((ny, nx - 1))
    q = np.zeros((ny - 1, nx))
    r, s = p.copy(), q.copy()
    t = 1.0

    def prox(v):
        if nonneg:
            return positive(v, box)
        return soft_threshold(v, lam_l1, box)

    for _ in range(iters):
        tnew = (1 + math.sqrt(1 + 4 * t * t)) / 2
        xv = prox(b - lam_tv * lpq(nx, ny, r, s))
        np_, nq_ = lx(nx, ny, xv)
        r = r + np_ / (8 * lam_tv)
        s = s + nq_ / (8 * lam_tv)
        np_, nq_ = p_pqiso(r, s)
        beta1 = 1 + (t - 1) / tnew
        beta2 = -(t - 1) / tnew
        r = np_ * beta1 + p * beta2
        s = nq_ * beta1 + q * beta2
        t = tnew
        p, q = np_, nq_
    return prox(b - lam_tv * lpq(nx, ny, p, q))


def q_part(xnew, z, c, dfdx):
    """calc_Q_part (c/mfista_tools.c:61-77)."""
    d = xnew - z
    return -(dfdx @ d) + c * (d @ d) / 2


# --------------------------------------------------------------------------
# the MFISTA loop (c/mfista_nufft_lib.c:308-553 TV, :557-787 TSV; the FFT and
# DFT libraries repeat the same loop: c/mfista_fft_lib.c:179-609,
# c/mfista_dft_lib.c:70-436)
# --------------------------------------------------------------------------

def mfista(f_part, grad, x0, nx, ny, maxiter, eps, lam_l1, lam_tv, lam_tsv, cinit,
           nonneg_flag, box_flag=0, cl_box=None, fgp_iter=FGPITER, trace=None, eta_first=None):
    """Returns (xout, iterations, c).  ``eps`` is the already-scaled threshold.

    TSV form when lam_tv == 0, TV form otherwise (the caller checks the
    both-positive error case).  ``trace`` (a list) collects per-iteration
    (cost, c) pairs when given.  ``eta_first``: the backtracking factor of
    the first outer iteration only (the C++ build uses 10,
    c++/mfista_nufft_lib.cpp:818, :860-863; the C library ETA throughout);
    the division after every backtracking loop stays ETA."""
    use_tv = lam_tv != 0
    box = np.asarray(cl_box) if box_flag == 1 else None
    x = np.array(x0, dtype=np.float64, copy=True)
    n = x.size
    if not use_tv and nonneg_flag not in (0, 1):
        return None, 0, cinit
    c = float(cinit)
    mu = 1.0

    def prox_tsv(v, eta):
        if nonneg_flag == 1:
            return soft_threshold_nonneg(v, eta, box)
        return soft_threshold(v, eta, box)

    z = x.copy()
    fx, _ = f_part(x)
    cost_now = fx + lam_l1 * np.abs(x).sum()
    if use_tv:
        cost_now += lam_tv * tv(nx, ny, x)
    elif lam_tsv > 0:
        cost_now += lam_tsv * tsv(nx, ny, x)
    cost = np.zeros(maxiter)
    it = 0
    xnew = x
    while it < maxiter:
        cost[it] = cost_now
        if trace is not None:
            trace.append((cost_now, c))
        qcore, resid = f_part(z)
        dfdx = grad(resid)
        if not use_tv and lam_tsv > 0:
            qcore += lam_tsv * tsv(nx, ny, z)
            dfdx = dfdx - lam_tsv * d_tsv(nx, ny, z)
        for _ in range(maxiter):
            if use_tv:
                if nonneg_flag == 1:
                    b = -lam_l1 / c + dfdx / c + z
                    xnew = fgp(nx, ny, b, 0.0, lam_tv / c, fgp_iter, True, box)
                else:
                    b = dfdx / c + z
                    xnew = fgp(nx, ny, b, lam_l1 / c, lam_tv / c, fgp_iter, False, box)
            else:
                xnew = prox_tsv(dfdx * (1.0 / c) + z, lam_l1 / c)
            fval, _ = f_part(xnew)
            if not use_tv and lam_tsv > 0:
                fval += lam_tsv * tsv(nx, ny, xnew)
            qval = q_part(xnew, z, c, dfdx) + qcore
            if fval <= qval:
                break
            c *= ETA if (eta_first is None or it > 0) else eta_first
        c /= ETA
        munew = (1 + math.sqrt(1 + 4 * mu * mu)) / 2
        fval += lam_l1 * np.abs(xnew).sum()
        if use_tv:
            fval += lam_tv * tv(nx, ny, xnew)
        if fval < cost[it]:
            cost_now = fval
            z = x * ((1 - mu) / munew) + xnew * (1 + (mu - 1) / munew)
            x = xnew.copy()
        else:
            z = x * (1 - mu / munew) + xnew * (mu / munew)
            if it > 1 and np.abs(x).sum() == 0:
                break
        if it >= MINITER and (cost[it - TD] - cost[it]) < eps:
            break
        mu = munew
        it += 1
    if it == maxiter:
        it -= 1
    return x, it + 1, c


# --------------------------------------------------------------------------
# entry points (c/mfista_nufft_lib.c:909-957, c/mfista_fft_lib.c:701-756,
# c/mfista_dft_lib.c:540-589) and result summaries (:791-905, :613-697,
# :440-536)
# --------------------------------------------------------------------------

def _summary(sq_error, m_report, m_div, x, nx, ny, lam_l1, lam_tv, lam_tsv):
    res = dict(M=m_report, N=nx * ny, NX=nx, NY=ny, lambda_l1=lam_l1, lambda_tv=lam_tv,
               lambda_tsv=lam_tsv, sq_error=sq_error, mean_sq_error=sq_error / m_div)
    ax = np.abs(x)
    res["l1cost"] = float(ax[ax > 0].sum())
    res["N_active"] = int(np.count_nonzero(ax > 0))
    fc = sq_error / 2
    if lam_l1 > 0:
        fc += lam_l1 * res["l1cost"]
    if lam_tsv > 0:
        res["tsvcost"] = tsv(nx, ny, x)
        fc += lam_tsv * res["tsvcost"]
    elif lam_tv > 0:
        res["tvcost"] = tv(nx, ny, x)
        fc += lam_tv * res["tvcost"]
    res["finalcost"] = fc
    return res


def _dispatch_ok(lam_tv, lam_tsv):
    return lam_tv == 0 or lam_tsv == 0


def imaging_core_nufft(u_dx, v_dy, vis_r, vis_i, vis_std, nx, ny, maxiter, eps,
                       lam_l1, lam_tv, lam_tsv, cinit, xinit, nonneg_flag, box_flag=0,
                       cl_box=None, fgp_iter=FGPITER, xout=None, trace=None):
    """mfista_imaging_core_nufft; returns (xout, result dict) or (None, None)
    when both lambda_tv and lambda_tsv are non-zero (:938-941)."""
    vis_r = np.asarray(vis_r, np.float64)
    vis_i = np.asarray(vis_i, np.float64)
    m = vis_r.size
    epsilon = (vis_r @ vis_r + vis_i @ vis_i) * eps / float(m)
    if not _dispatch_ok(lam_tv, lam_tsv):
        return None, None
    plan = NufftPlan(u_dx, v_dy, nx, ny)
    w = 1.0 / np.asarray(vis_std, np.float64)
    fp = lambda x: nufft_f_part(plan, vis_r, vis_i, w, x)
    gr = lambda r: nufft_grad(plan, w, r)
    x, it, c = mfista(fp, gr, xinit, nx, ny, maxiter, epsilon, lam_l1, lam_tv, lam_tsv,
                      cinit, nonneg_flag, box_flag, cl_box, fgp_iter, trace)
    if x is None:   # bad nonneg flag: xout is left as the caller passed it (:634-637)
        x = np.zeros(nx * ny) if xout is None else np.asarray(xout, np.float64)
    chi, _ = fp(x)
    res = _summary(2 * chi, m // 2, m, x, nx, ny, lam_l1, lam_tv, lam_tsv)
    res.update(ITER=it, nonneg=nonneg_flag, Lip_const=c, maxiter=maxiter)
    return x, res


def imaging_core_fft(u_idx, v_idx, y_r, y_i, noise, nx, ny, maxiter, eps, lam_l1,
                     lam_tv, lam_tsv, cinit, xinit, nonneg_flag, box_flag=0, cl_box=None,
                     fgp_iter=FGPITER, xout=None, trace=None):
    """mfista_imaging_core_fft (c/mfista_fft_lib.c:701-756)."""
    y_r = np.asarray(y_r, np.float64)
    y_i = np.asarray(y_i, np.float64)
    m = y_r.size
    epsilon = float(np.sum(y_r * y_r + y_i * y_i)) * eps / float(m)
    if not _dispatch_ok(lam_tv, lam_tsv):
        return None, None
    op = FftOperator(u_idx, v_idx, y_r, y_i, noise, nx, ny)
    x, it, c = mfista(op.f_part, op.grad, xinit, nx, ny, maxiter, epsilon, lam_l1, lam_tv,
                      lam_tsv, cinit, nonneg_flag, box_flag, cl_box, fgp_iter, trace)
    if x is None:
        x = np.zeros(nx * ny) if xout is None else np.asarray(xout, np.float64)
    chi, _ = op.f_part(x)
    res = _summary(2 * chi, m // 2, m, x, nx, ny, lam_l1, lam_tv, lam_tsv)
    res.update(ITER=it, nonneg=nonneg_flag, Lip_const=c, maxiter=maxiter)
    return x, res


def imaging_core_dft(y, A, nx, ny, maxiter, eps, lam_l1, lam_tv, lam_tsv, cinit, xinit,
                     nonneg_flag, box_flag=0, cl_box=None, fgp_iter=FGPITER, trace=None):
    """mfista_imaging_core_dft (c/mfista_dft_lib.c:540-589); eps is used raw."""
    op = DftOperator(y, A)
    xin = np.array(xinit, np.float64, copy=True)
    if not _dispatch_ok(lam_tv, lam_tsv):
        return None, None
    x, it, c = mfista(op.f_part, op.grad, xin, nx, ny, maxiter, eps, lam_l1, lam_tv,
                      lam_tsv, cinit, nonneg_flag, box_flag, cl_box, fgp_iter, trace)
    if x is None:
        x = xin
    chi, r = op.f_part(x)
    res = _summary(2 * chi, op.y.size, op.y.size, x, nx, ny, lam_l1, lam_tv, lam_tsv)
    res.update(ITER=it, nonneg=nonneg_flag, Lip_const=c, maxiter=maxiter, residual=r)
    return x, res


def lipschitz_nufft(plan, weight, iters=30, seed=0):
    """Power-iteration estimate of the Lipschitz constant of the chi^2
    gradient (A^H W^2 A), used to pick ``cinit`` for seeded fixtures."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(plan.nx * plan.ny)
    lam = 0.0
    for _ in range(iters):
        x /= np.linalg.norm(x)
        fr, fi = plan.forward(x)
        y = plan.adjoint(fr * weight * weight, fi * weight * weight)
        lam = float(x @ y)
        x = y
    return lam
