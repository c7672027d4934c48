"""CPU oracle of the C++ build's NUFFT operators (test infrastructure only).

TEST INFRASTRUCTURE ONLY: `tests/` use it as the checker; the library never
calls it.

The reference ships a second build (c++/, exporting the same C names plus
x2y_nufft / y2x_nufft, c++/mfista.hpp:136-140) whose NUFFT differs from the
C library's: MSP = 6 (12 taps per axis, c++/mfista.hpp:32-35), floor binning
of points flipped to v >= 0, one Gaussian width tau = MSP / Nx^2 for both
axes, the E3 factor folded into E2, and Hermitian halos in padded buffers.
Restated here from c++/mfista_nufft_lib.cpp:

* preNUFFT (:85-187): per point y_neg = v < 0 (u, v negated then),
  m = floor(u 2N / 2 pi), xi = 2 pi m / 2N, E1 = exp(-(u-xi_x)^2/4tau
  - (v-xi_y)^2/4tau), E2[j] = exp(c_j (pi (u-xi)/(2N tau) - c_j pi^2 /
  ((2N)^2 tau))) with c_j = j - MSP + 1, E4[i, j] = (Nx Ny pi / MSP)
  exp(tau (i - Nx/2)^2 + tau (j - Ny/2)^2);
* NUFFT2d2 (:440-504, forward): x E4 padded with the image centre at the
  origin of the 2Nx x 2Ny grid (small2large :46-77), real-to-complex FFT,
  the half plane copied into a buffer with MSP-wide halos whose ky < 0 rows
  are the Hermitian images of ky > 0 (kx from 1-Nx to Nx-1), then per point
  Fout = conj(E1 sum_ab E2y_a E2x_b G(mx + c_b, my + c_a)) / (4 Nx Ny),
  conjugated again for y_neg points;
* NUFFT2d1_sngl (:189-258, adjoint): conj(Fin) (Fin for y_neg points) times
  E1 / (8 Nx Ny) scattered into a buffer with the same halos, the ky < 0
  halo, the kx = -Nx row, and the ky = 0 and ky = Ny columns folded back as
  conjugates, the DC cell doubled, complex-to-real FFT, unpadded times E4
  (large2small :18-44).
Taps that fall outside the halos are dropped, as there (the reference warns
when points come within MSP of the grid edge, :155-156, :180-185).

The C++ sources need Eigen, which is not in this image, so this restatement
cannot be checked against the compiled reference here; it is pinned by the
transform it approximates (the exact DFT, to the accuracy of a 12-tap
kernel) and by adjointness of the two operators
(tests/test_cpp_nufft_oracle.py).
"""
from __future__ import annotations

import math

import numpy as np

MSP = 6
MSP2 = 2 * MSP


class CppNufftPlan:
    def __init__(self, u, v, nx, ny):
        u = np.asarray(u, np.float64)
        v = np.asarray(v, np.float64)
        self.nx, self.ny, self.m = nx, ny, u.size
        self.y_neg = v < 0
        uk = np.where(self.y_neg, -u, u)
        vk = np.where(self.y_neg, -v, v)
        mrx, mry = 2.0 * nx, 2.0 * ny
        tau = MSP / float(nx * nx)
        coeff = float(nx * ny) * math.pi / MSP
        t3x = math.pi * math.pi / (mrx * mrx * tau)
        t3y = math.pi * math.pi / (mry * mry * tau)
        c = np.arange(MSP2, dtype=np.float64) - MSP + 1
        self.mx = np.floor(uk * mrx / (2 * math.pi)).astype(np.int64)
        self.my = np.floor(vk * mry / (2 * math.pi)).astype(np.int64)
        xix = 2 * math.pi * self.mx / mrx
        xiy = 2 * math.pi * self.my / mry
        self.e1 = np.exp(-((uk - xix) ** 2) / (4 * tau) - ((vk - xiy) ** 2) / (4 * tau))
        t4x = math.pi * (uk - xix) / (mrx * tau)
        t4y = math.pi * (vk - xiy) / (mry * tau)
        self.e2x = np.exp(c[None, :] * (t4x[:, None] - c[None, :] * t3x))   # [M][12]
        self.e2y = np.exp(c[None, :] * (t4y[:, None] - c[None, :] * t3y))
        ti = (np.arange(nx) - nx // 2).astype(np.float64)
        tj = (np.arange(ny) - ny // 2).astype(np.float64)
        self.e4 = coeff * np.exp(tau * ti[:, None] ** 2 + tau * tj[None, :] ** 2)
        # padded position of image pixel (i, j): the centre at the origin
        self.pr = (np.arange(nx) - nx // 2) % (2 * nx)
        self.pc = (np.arange(ny) - ny // 2) % (2 * ny)
        # tap cells: buffer rows / columns of the 12 x 12 block of each point
        a = np.arange(MSP2)
        self.hy = self.my[:, None] + 1 + a[None, :]           # forward buffer rows (ky + MSP)
        self.hx = self.mx[:, None] + nx + 1 + a[None, :]      # forward buffer cols (kx + Nx + MSP)

    def forward(self, x):
        """x2y_nufft: (real, imag) of A x."""
        nx, ny = self.nx, self.ny
        x = np.asarray(x, np.float64).reshape(nx, ny)
        P = np.zeros((2 * nx, 2 * ny))
        P[np.ix_(self.pr, self.pc)] = x * self.e4
        G = np.fft.rfft2(P)                                   # (2nx, ny+1)
        H = np.zeros((ny + 1 + MSP2, 2 * nx + MSP2), complex)
        for kx in range(-nx, nx):
            H[MSP:MSP + ny + 1, kx + nx + MSP] = G[kx % (2 * nx), :]
        for i in range(MSP):                                  # ky = i - MSP < 0
            for kx in range(1 - nx, nx):
                H[i, kx + nx + MSP] = np.conj(H[MSP2 - i, -kx + nx + MSP])
        blk = H[self.hy[:, :, None], self.hx[:, None, :]]     # [M][12 y][12 x]
        s = np.einsum("ka,kb,kab->k", self.e2y, self.e2x, blk)
        f = np.conj(s) * self.e1 / (4.0 * nx * ny)
        f = np.where(self.y_neg, np.conj(f), f)
        return f.real.copy(), f.imag.copy()

    def adjoint(self, yr, yi):
        """y2x_nufft: the image from visibilities (real, imag)."""
        nx, ny = self.nx, self.ny
        fin = np.asarray(yr, np.float64) + 1j * np.asarray(yi, np.float64)
        vis = np.where(self.y_neg, fin, np.conj(fin))
        v0 = vis * self.e1 / (8.0 * nx * ny)
        L = np.zeros((2 * nx + MSP2, ny + 1 + MSP2), complex)  # rows kx + Nx + MSP, cols ky + MSP
        w = v0[:, None, None] * self.e2x[:, :, None] * self.e2y[:, None, :]
        np.add.at(L, (self.hx[:, :, None], self.hy[:, None, :]), w)
        # ky < 0 halo folded back as conjugates (rows kx = 0..Nx-1, then 1-Nx..-1)
        L[MSP + nx:MSP + 2 * nx, MSP + 1:MSP2 + 1] += np.conj(L[MSP + 1:MSP + nx + 1, 0:MSP][::-1, ::-1])
        L[MSP + 1:MSP + nx, MSP + 1:MSP2 + 1] += np.conj(L[MSP + nx + 1:MSP + 2 * nx, 0:MSP][::-1, ::-1])
        # kx = -Nx row
        L[MSP, MSP + 1:MSP2] += np.conj(L[MSP, 1:MSP][::-1])
        # ky = 0 and ky = Ny columns: kx and -kx folded onto each other
        for col in (MSP, MSP + ny):
            buf = L[MSP:MSP + 2 * nx, col].copy()
            L[MSP + nx + 1:MSP + 2 * nx, col] += np.conj(buf[1:nx][::-1])
            L[MSP + 1:MSP + nx, col] += np.conj(buf[nx + 1:2 * nx][::-1])
        L[MSP + nx, MSP] *= 2.0
        C = np.zeros((2 * nx, ny + 1), complex)
        C[:nx] = L[MSP + nx:MSP + 2 * nx, MSP:MSP + ny + 1]
        C[nx:] = L[MSP:MSP + nx, MSP:MSP + ny + 1]
        out = np.fft.irfft2(C, s=(2 * nx, 2 * ny)) * (4.0 * nx * ny)
        return (out[np.ix_(self.pr, self.pc)] * self.e4).ravel()


def cpp_imaging_core_nufft(u_dx, v_dy, vis_r, vis_i, vis_std, nx, ny, maxiter, eps, lam_l1, lam_tsv, cinit,
                           xinit, nonneg_flag):
    """The C++ build's mfista_imaging_core_nufft, TSV form
    (c++/mfista_nufft_lib.cpp:680-929, :1016-1074): the C library's loop
    with these operators and a backtracking factor of 10 in the first
    iteration.  Returns (xout, iterations, final c).  The C++ build also
    sorts the caller's u, v, vis arrays in place (sort_input :550-641); the
    sums here do not depend on the order beyond rounding, so it is left
    out.  eps is scaled as in the C library (:1031-1034)."""
    from . import mfista_oracle as R
    vis_r = np.asarray(vis_r, np.float64)
    vis_i = np.asarray(vis_i, np.float64)
    m = vis_r.size
    epsilon = (vis_r @ vis_r + vis_i @ vis_i) * eps / float(m)
    plan = CppNufftPlan(u_dx, v_dy, nx, ny)
    w = 1.0 / np.asarray(vis_std, np.float64)

    def f_part(x):
        fr, fi = plan.forward(x)
        rr = (vis_r - fr) * w
        ri = (vis_i - fi) * w
        return 0.5 * (rr @ rr + ri @ ri), (rr, ri)

    def grad(res):
        rr, ri = res
        return plan.adjoint(rr * w, ri * w)

    return R.mfista(f_part, grad, xinit, nx, ny, maxiter, epsilon, lam_l1, 0.0, lam_tsv, cinit, nonneg_flag,
                    eta_first=10.0)
