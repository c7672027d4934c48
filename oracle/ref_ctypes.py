"""ctypes binding to the reference C solvers compiled unchanged into
oracle/_ref/libmfista_ref.so (see oracle/Makefile).

TEST INFRASTRUCTURE ONLY: used by tests/ and tests/golden/make_golden.py to
pin the numpy restatement (oracle/mfista_oracle.py) against the reference
itself, and by bench.py's reference arm.  The library exports the
reference's internal functions as well as its entry points, so single
operators (preNUFFT, NUFFT2d1/2d2, TSV, FGP ...) can be called directly.
"""
from __future__ import annotations

import ctypes as C
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_fp = C.POINTER(C.c_float)


class RESULT(C.Structure):
    """struct RESULT, c/mfista.h:45-66."""
    _fields_ = [("M", C.c_int), ("N", C.c_int), ("NX", C.c_int), ("NY", C.c_int),
                ("N_active", C.c_int), ("maxiter", C.c_int), ("ITER", C.c_int),
                ("nonneg", C.c_int), ("lambda_l1", C.c_double), ("lambda_tv", C.c_double),
                ("lambda_tsv", C.c_double), ("sq_error", C.c_double),
                ("mean_sq_error", C.c_double), ("l1cost", C.c_double), ("tvcost", C.c_double),
                ("tsvcost", C.c_double), ("finalcost", C.c_double), ("comp_time", C.c_double),
                ("residual", _dp), ("Lip_const", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "residual"}


_libs = {}


def available(fgp50=False):
    return os.path.exists(_path(fgp50))


def _path(fgp50):
    return os.path.join(REF_DIR, "libmfista_ref_fgp50.so" if fgp50 else "libmfista_ref.so")


def load(fgp50=False):
    key = bool(fgp50)
    if key not in _libs:
        lib = C.CDLL(_path(fgp50))
        lib.fftw_plan_dft_r2c_2d.restype = C.c_void_p
        lib.fftw_plan_dft_r2c_2d.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_uint]
        lib.fftw_plan_dft_c2r_2d.restype = C.c_void_p
        lib.fftw_plan_dft_c2r_2d.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_uint]
        lib.fftw_destroy_plan.argtypes = [C.c_void_p]
        for name in ("TSV", "TV"):
            getattr(lib, name).restype = C.c_double
        lib.calc_F_part_nufft.restype = C.c_double
        lib.calc_Q_part.restype = C.c_double
        _libs[key] = lib
    return _libs[key]


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _i(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return a, a.ctypes.data_as(_ip)


def _f(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(_fp)


class RefNufft:
    """preNUFFT + FFTW-shim plans, for calling NUFFT2d1 / NUFFT2d2 directly."""

    def __init__(self, u, v, nx, ny):
        lib = self.lib = load()
        m = len(u)
        self.m, self.nx, self.ny = m, nx, ny
        self.E1 = np.zeros(m)
        self.E2x = np.zeros(24 * m)
        self.E2y = np.zeros(24 * m)
        self.E3x = np.zeros(13)
        self.E3y = np.zeros(13)
        self.E4 = np.zeros(nx * ny)
        self.mx = np.zeros(m, np.int32)
        self.my = np.zeros(m, np.int32)
        self._u, pu = _d(u)
        self._v, pv = _d(v)
        lib.preNUFFT(self.E1.ctypes.data_as(_dp), self.E2x.ctypes.data_as(_dp),
                     self.E2y.ctypes.data_as(_dp), self.E3x.ctypes.data_as(_dp),
                     self.E3y.ctypes.data_as(_dp), self.E4.ctypes.data_as(_dp),
                     self.mx.ctypes.data_as(_ip), self.my.ctypes.data_as(_ip), pu, pv,
                     C.c_int(m), C.c_int(nx), C.c_int(ny))
        self.rvec = np.zeros(4 * nx * ny)
        self.cvec = np.zeros(2 * nx * (ny + 1), np.complex128)
        self.p_r2c = C.c_void_p(lib.fftw_plan_dft_r2c_2d(2 * nx, 2 * ny, self.rvec.ctypes.data,
                                                         self.cvec.ctypes.data, 0))
        self.p_c2r = C.c_void_p(lib.fftw_plan_dft_c2r_2d(2 * nx, 2 * ny, self.cvec.ctypes.data,
                                                         self.rvec.ctypes.data, 0))

    def _geom(self):
        return (C.c_int(self.m), C.c_int(self.nx), C.c_int(self.ny),
                self.E1.ctypes.data_as(_dp), self.E2x.ctypes.data_as(_dp),
                self.E2y.ctypes.data_as(_dp), self.E3x.ctypes.data_as(_dp),
                self.E3y.ctypes.data_as(_dp), self.E4.ctypes.data_as(_dp),
                self.mx.ctypes.data_as(_ip), self.my.ctypes.data_as(_ip))

    def forward(self, x):
        fr = np.zeros(self.m)
        fi = np.zeros(self.m)
        xx, px = _d(x)
        self.rvec[:] = 0.0
        self.lib.NUFFT2d2(fr.ctypes.data_as(_dp), fi.ctypes.data_as(_dp), *self._geom(),
                          self.rvec.ctypes.data_as(_dp), C.c_void_p(self.cvec.ctypes.data),
                          C.byref(self.p_r2c), px)
        return fr, fi

    def adjoint(self, r_r, r_i):
        X = np.zeros(self.nx * self.ny)
        a, pa = _d(r_r)
        b, pb = _d(r_i)
        self.lib.NUFFT2d1(X.ctypes.data_as(_dp), *self._geom(), C.c_void_p(self.cvec.ctypes.data),
                          self.rvec.ctypes.data_as(_dp), C.byref(self.p_c2r), pa, pb)
        return X

    def close(self):
        self.lib.fftw_destroy_plan(self.p_r2c)
        self.lib.fftw_destroy_plan(self.p_c2r)


def tsv(nx, ny, x):
    xx, p = _d(x)
    return load().TSV(C.c_int(nx), C.c_int(ny), p)


def d_tsv(nx, ny, x):
    xx, p = _d(x)
    out = np.zeros(nx * ny)
    load().d_TSV(C.c_int(nx), C.c_int(ny), p, out.ctypes.data_as(_dp))
    return out


def tv(nx, ny, x):
    xx, p = _d(x)
    return load().TV(C.c_int(nx), C.c_int(ny), p)


def fgp(nx, ny, b, lam_l1, lam_tv, iters, nonneg, box=None):
    """FGP_L1_box / FGP_nonneg_box (c/mfista_TV_lib.c:189-384)."""
    lib = load()
    n = nx * ny
    nn = C.c_int(n)
    bb, pb = _d(b)
    mats = [np.zeros(n) for _ in range(6)]
    ptrs = [m.ctypes.data_as(_dp) for m in mats]
    out = np.zeros(n)
    box_flag = 0 if box is None else 1
    bx, pbx = _f(np.ones(n) if box is None else box)
    if nonneg:
        lib.FGP_nonneg_box(C.byref(nn), C.c_int(nx), C.c_int(ny), pb, C.c_double(lam_tv),
                           C.c_int(iters), *ptrs, out.ctypes.data_as(_dp), C.c_int(box_flag), pbx)
    else:
        lib.FGP_L1_box(C.byref(nn), C.c_int(nx), C.c_int(ny), pb, C.c_double(lam_l1),
                       C.c_double(lam_tv), C.c_int(iters), *ptrs, out.ctypes.data_as(_dp),
                       C.c_int(box_flag), pbx)
    return out


def _box(n, cl_box):
    if cl_box is None:
        return _f(np.ones(n))
    return _f(cl_box)


def core_nufft(u, v, vis_r, vis_i, vis_std, nx, ny, maxiter, eps, lam_l1, lam_tv, lam_tsv,
               cinit, xinit=None, nonneg_flag=1, box_flag=0, cl_box=None, fgp50=False,
               xout_init=None):
    lib = load(fgp50)
    n = nx * ny
    keep = [_d(u), _d(v), _d(vis_r), _d(vis_i), _d(vis_std)]
    xi, pxi = _d(np.zeros(n) if xinit is None else xinit)
    xo = np.zeros(n) if xout_init is None else np.array(xout_init, np.float64, copy=True)
    bx, pbx = _box(n, cl_box)
    res = RESULT()
    lib.mfista_imaging_core_nufft(*[k[1] for k in keep], C.c_int(len(u)), C.c_int(nx),
                                  C.c_int(ny), C.c_int(maxiter), C.c_double(eps),
                                  C.c_double(lam_l1), C.c_double(lam_tv), C.c_double(lam_tsv),
                                  C.c_double(cinit), pxi, xo.ctypes.data_as(_dp),
                                  C.c_int(nonneg_flag), C.c_int(box_flag), pbx, C.byref(res))
    return xo, res


def core_fft(u_idx, v_idx, y_r, y_i, noise, nx, ny, maxiter, eps, lam_l1, lam_tv, lam_tsv,
             cinit, xinit=None, nonneg_flag=1, box_flag=0, cl_box=None, fgp50=False,
             xout_init=None):
    lib = load(fgp50)
    n = nx * ny
    ui, pu = _i(u_idx)
    vi, pv = _i(v_idx)
    keep = [_d(y_r), _d(y_i), _d(noise)]
    xi, pxi = _d(np.zeros(n) if xinit is None else xinit)
    xo = np.zeros(n) if xout_init is None else np.array(xout_init, np.float64, copy=True)
    bx, pbx = _box(n, cl_box)
    res = RESULT()
    lib.mfista_imaging_core_fft(pu, pv, *[k[1] for k in keep], C.c_int(len(u_idx)), C.c_int(nx),
                                C.c_int(ny), C.c_int(maxiter), C.c_double(eps),
                                C.c_double(lam_l1), C.c_double(lam_tv), C.c_double(lam_tsv),
                                C.c_double(cinit), pxi, xo.ctypes.data_as(_dp),
                                C.c_int(nonneg_flag), C.c_uint(64), C.c_int(box_flag), pbx,
                                C.byref(res))
    return xo, res


def core_dft(y, A, nx, ny, maxiter, eps, lam_l1, lam_tv, lam_tsv, cinit, xinit=None,
             nonneg_flag=1, box_flag=0, cl_box=None, fgp50=False):
    """A is the logical (M, N) matrix; it is passed column-major as the reference expects."""
    lib = load(fgp50)
    A = np.asarray(A, np.float64)
    m, n = A.shape
    Af = np.asfortranarray(A)
    yy, py = _d(y)
    xi, pxi = _d(np.zeros(n) if xinit is None else xinit)
    xo = np.zeros(n)
    bx, pbx = _box(n, cl_box)
    mm = C.c_int(m)
    nn = C.c_int(n)
    res = RESULT()
    lib.mfista_imaging_core_dft(py, Af.ctypes.data_as(_dp), C.byref(mm), C.byref(nn), C.c_int(nx),
                                C.c_int(ny), C.c_int(maxiter), C.c_double(eps),
                                C.c_double(lam_l1), C.c_double(lam_tv), C.c_double(lam_tsv),
                                C.c_double(cinit), pxi, xo.ctypes.data_as(_dp),
                                C.c_int(nonneg_flag), C.c_int(0), C.c_int(box_flag), pbx,
                                C.byref(res))
    resid = None
    if res.ITER > 0 and bool(res.residual):
        resid = np.ctypeslib.as_array(res.residual, shape=(m,)).copy()
    return xo, res, resid
