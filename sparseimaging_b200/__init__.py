"""B200 (sm_100a) MFISTA sparse-imaging solver.

Python binding of libmfista_b200.so.  The raw functions
``mfista_imaging_core_nufft/fft/dft`` take the reference's arguments in the
reference's order (c/mfista.h:151-178) and write ``xout`` and a ``RESULT``
in place, like the C entry points; ``imaging_core_*`` are convenience
wrappers returning ``(xout, result_dict)``.  The extensions (batched solves,
device-resident plans, operator calls) are wrapped below them.

The library is the only compute path: if it is not built, or a call fails on
the GPU, these functions raise; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .build import LIB

__all__ = ["RESULT", "Problem", "MfistaError", "lib", "mfista_imaging_core_nufft",
           "mfista_imaging_core_fft", "mfista_imaging_core_dft", "imaging_core_nufft",
           "imaging_core_fft", "imaging_core_dft", "nufft_batch", "fft_batch", "fgp_profile", "dft_batch", "Plan", "nufft_forward",
           "nufft_adjoint", "fgp_prox", "nufft_lipschitz", "last_status", "last_error", "set_fgp_iter", "set_device",
           "dft_apply", "dft_profile", "cpp_x2y_nufft", "cpp_y2x_nufft", "cpp_imaging_core_nufft", "FP64", "FP32", "BF16X3", "BF16X6"]

FP64 = 64
FP32 = 32
BF16X3 = 3  # DFT only: tensor-core split-BF16 products (2 planes, 3 products) with FP64 anchor correction
BF16X6 = 6  # DFT only: 3 planes, 6 products (~FP32 accuracy) with FP64 anchor correction

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_fp = C.POINTER(C.c_float)


class RESULT(C.Structure):
    """struct RESULT (c/mfista.h:45-66); byte-identical layout."""
    _fields_ = [("M", C.c_int), ("N", C.c_int), ("NX", C.c_int), ("NY", C.c_int),
                ("N_active", C.c_int), ("maxiter", C.c_int), ("ITER", C.c_int),
                ("nonneg", C.c_int), ("lambda_l1", C.c_double), ("lambda_tv", C.c_double),
                ("lambda_tsv", C.c_double), ("sq_error", C.c_double),
                ("mean_sq_error", C.c_double), ("l1cost", C.c_double), ("tvcost", C.c_double),
                ("tsvcost", C.c_double), ("finalcost", C.c_double), ("comp_time", C.c_double),
                ("residual", _dp), ("Lip_const", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "residual"}


class Problem(C.Structure):
    """struct mfista_problem (include/mfista_b200.h)."""
    _fields_ = [("lambda_l1", C.c_double), ("lambda_tv", C.c_double),
                ("lambda_tsv", C.c_double), ("cinit", C.c_double), ("maxiter", C.c_int),
                ("nonneg_flag", C.c_int), ("target_cost", C.c_double)]


class MfistaError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"mfista status {status}: {msg}")
        self.status = status


_lib = None


def lib():
    """Loads libmfista_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError(f"{LIB} is not built; run `python -m sparseimaging_b200.build`")
        L = C.CDLL(LIB)
        L.mfista_last_error.restype = C.c_char_p
        L.mfista_last_status.restype = C.c_int
        L.mfista_set_device.restype = C.c_int
        L.mfista_set_device.argtypes = [C.c_int]
        L.mfista_set_fgp_iter.restype = C.c_int
        L.mfista_set_fgp_iter.argtypes = [C.c_int]
        L.mfista_imaging_core_nufft.restype = None
        L.mfista_imaging_core_nufft.argtypes = [_dp, _dp, _dp, _dp, _dp, C.c_int, C.c_int, C.c_int,
                                                C.c_int, C.c_double, C.c_double, C.c_double,
                                                C.c_double, C.c_double, _dp, _dp, C.c_int, C.c_int,
                                                _fp, C.POINTER(RESULT)]
        L.mfista_imaging_core_fft.restype = None
        L.mfista_imaging_core_fft.argtypes = [_ip, _ip, _dp, _dp, _dp, C.c_int, C.c_int, C.c_int,
                                              C.c_int, C.c_double, C.c_double, C.c_double,
                                              C.c_double, C.c_double, _dp, _dp, C.c_int, C.c_uint,
                                              C.c_int, _fp, C.POINTER(RESULT)]
        L.mfista_imaging_core_dft.restype = None
        L.mfista_imaging_core_dft.argtypes = [_dp, _dp, _ip, _ip, C.c_int, C.c_int, C.c_int,
                                              C.c_double, C.c_double, C.c_double, C.c_double,
                                              C.c_double, _dp, _dp, C.c_int, C.c_int, C.c_int, _fp,
                                              C.POINTER(RESULT)]
        L.mfista_nufft_batch.restype = C.c_int
        L.mfista_nufft_batch.argtypes = [_dp, _dp, _dp, _dp, _dp, _ip, C.c_int, C.c_int, C.c_int,
                                         C.c_int, C.c_int, C.POINTER(Problem), C.c_double, C.c_int,
                                         C.c_int, _dp, _dp, C.POINTER(RESULT)]
        L.mfista_fft_batch.restype = C.c_int
        L.mfista_fft_batch.argtypes = [_ip, _ip, _dp, _dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.POINTER(Problem), C.c_double, C.c_int, C.c_int, _dp, _dp,
                                       C.POINTER(RESULT)]
        L.mfista_fgp_profile.restype = C.c_int
        L.mfista_fgp_profile.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp]
        L.mfista_dft_batch.restype = C.c_int
        L.mfista_dft_batch.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.POINTER(Problem), C.c_double, C.c_int, C.c_int, _dp, _dp,
                                       C.POINTER(RESULT)]
        L.mfista_nufft_plan_create.restype = C.c_void_p
        L.mfista_nufft_plan_create.argtypes = [_dp, _dp, _dp, _dp, _dp, _ip, C.c_int, C.c_int,
                                               C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.mfista_plan_set_problems.restype = C.c_int
        L.mfista_plan_set_problems.argtypes = [C.c_void_p, C.POINTER(Problem), C.c_double, _dp]
        L.mfista_plan_run.restype = C.c_int
        L.mfista_plan_run.argtypes = [C.c_void_p]
        L.mfista_plan_fetch.restype = C.c_int
        L.mfista_plan_fetch.argtypes = [C.c_void_p, _dp, C.POINTER(RESULT)]
        L.mfista_plan_stream.restype = C.c_void_p
        L.mfista_plan_stream.argtypes = [C.c_void_p]
        L.mfista_plan_statuses.restype = C.c_int
        L.mfista_plan_statuses.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        L.mfista_plan_device_loop.restype = C.c_int
        L.mfista_plan_device_loop.argtypes = [C.c_void_p]
        L.mfista_plan_kernel_launches.restype = C.c_int
        L.mfista_plan_kernel_launches.argtypes = [C.c_void_p]
        L.mfista_plan_profile.restype = C.c_int
        L.mfista_plan_profile.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp]
        _i4 = C.POINTER(C.c_int)
        L.mfista_plan_get_shapes.restype = C.c_int
        L.mfista_plan_get_shapes.argtypes = [C.c_void_p, _i4]
        L.mfista_plan_set_shapes.restype = C.c_int
        L.mfista_plan_set_shapes.argtypes = [C.c_void_p, _i4]
        L.mfista_plan_tune.restype = C.c_int
        L.mfista_plan_tune.argtypes = [C.c_void_p, C.c_int, _i4, _dp]
        L.mfista_dft_apply.restype = C.c_int
        L.mfista_dft_apply.argtypes = [_dp, C.c_int, C.c_int, _dp, C.c_int, C.c_int, C.c_int, _dp]
        L.mfista_dft_profile.restype = C.c_int
        L.mfista_dft_profile.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp]
        L.mfista_release_cache.restype = None
        L.mfista_release_cache.argtypes = []
        L.mfista_nufft_movie.restype = C.c_int
        L.mfista_nufft_movie.argtypes = [_dp, _dp, _dp, _dp, _dp, _ip, C.c_int, C.c_int, C.c_int, _dp, C.c_double,
                                         C.c_double, C.c_double, C.c_double, C.c_int, C.c_double, C.c_int, _dp,
                                         C.c_int, _dp, _dp, C.POINTER(RESULT), _dp]
        L.mfista_cpp_y2x_nufft.restype = C.c_int
        L.mfista_cpp_y2x_nufft.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp]
        L.mfista_cpp_imaging_core_nufft.restype = None
        L.mfista_cpp_imaging_core_nufft.argtypes = L.mfista_imaging_core_nufft.argtypes
        L.mfista_cpp_imaging_core_fft.restype = None
        L.mfista_cpp_imaging_core_fft.argtypes = L.mfista_imaging_core_fft.argtypes
        L.mfista_cpp_x2y_nufft.restype = C.c_int
        L.mfista_cpp_x2y_nufft.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp]
        L.mfista_dft_looe.restype = C.c_int
        L.mfista_dft_looe.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_int, _dp, C.c_int, _dp, _dp, _dp, _ip]
        L.mfista_plan_destroy.restype = None
        L.mfista_plan_destroy.argtypes = [C.c_void_p]
        L.mfista_nufft_forward.restype = C.c_int
        L.mfista_nufft_forward.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.c_int]
        L.mfista_nufft_adjoint.restype = C.c_int
        L.mfista_nufft_adjoint.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.c_int]
        L.mfista_fgp_prox.restype = C.c_int
        L.mfista_fgp_prox.argtypes = [_dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                      C.c_int, _fp, _dp, C.c_int]
        L.mfista_nufft_lipschitz.restype = C.c_int
        L.mfista_nufft_lipschitz.argtypes = [_dp, _dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int, _dp]
        _lib = L
    return _lib


def set_device(device):
    """CUDA device for this thread's subsequent calls."""
    _check(lib().mfista_set_device(int(device)))


def release_cache():
    """Free the solvers mfista_imaging_core_nufft keeps between calls."""
    lib().mfista_release_cache()


def set_fgp_iter(n):
    """FGP iterations of the TV form in the drop-in calls (reference: 100)."""
    old = lib().mfista_set_fgp_iter(int(n))
    if old < 0:
        raise ValueError("fgp iterations must be >= 1")
    return old


def last_status():
    return lib().mfista_last_status()


def last_error():
    return lib().mfista_last_error().decode()


def _check(st=None):
    st = last_status() if st is None else st
    if st != 0:
        raise MfistaError(st, last_error())


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a, t=_dp):
    return None if a is None else a.ctypes.data_as(t)


# ---------------------------------------------------------------------------
# reference entry points, argument for argument
# ---------------------------------------------------------------------------

def mfista_imaging_core_nufft(u_dx, v_dy, vis_r, vis_i, vis_std, M, NX, NY, maxiter, eps,
                              lambda_l1, lambda_tv, lambda_tsv, cinit, xinit, xout, nonneg_flag,
                              box_flag, cl_box, mfista_result):
    """c/mfista.h:172-178.  Arrays must be float64 (cl_box float32) and
    contiguous; xout and mfista_result are written in place."""
    lib().mfista_imaging_core_nufft(_p(u_dx), _p(v_dy), _p(vis_r), _p(vis_i), _p(vis_std), M, NX,
                                    NY, maxiter, eps, lambda_l1, lambda_tv, lambda_tsv, cinit,
                                    _p(xinit), _p(xout), nonneg_flag, box_flag, _p(cl_box, _fp),
                                    C.byref(mfista_result))


def mfista_imaging_core_fft(u_idx, v_idx, y_r, y_i, noise_stdev, M, NX, NY, maxiter, eps,
                            lambda_l1, lambda_tv, lambda_tsv, cinit, xinit, xout, nonneg_flag,
                            fftw_plan_flag, box_flag, cl_box, mfista_result):
    """c/mfista.h:161-168."""
    lib().mfista_imaging_core_fft(_p(u_idx, _ip), _p(v_idx, _ip), _p(y_r), _p(y_i), _p(noise_stdev),
                                  M, NX, NY, maxiter, eps, lambda_l1, lambda_tv, lambda_tsv, cinit,
                                  _p(xinit), _p(xout), nonneg_flag, fftw_plan_flag, box_flag,
                                  _p(cl_box, _fp), C.byref(mfista_result))


def mfista_imaging_core_dft(y, A, M, N, NX, NY, maxiter, eps, lambda_l1, lambda_tv, lambda_tsv,
                            cinit, xinit, xout, nonneg_flag, looe_flag, box_flag, cl_box,
                            mfista_result):
    """c/mfista.h:151-157 (M and N are ctypes ints passed by reference)."""
    lib().mfista_imaging_core_dft(_p(y), _p(A), C.byref(M), C.byref(N), NX, NY, maxiter, eps,
                                  lambda_l1, lambda_tv, lambda_tsv, cinit, _p(xinit), _p(xout),
                                  nonneg_flag, looe_flag, box_flag, _p(cl_box, _fp),
                                  C.byref(mfista_result))


# ---------------------------------------------------------------------------
# convenience wrappers
# ---------------------------------------------------------------------------

def _box(n, cl_box):
    return np.ones(n, np.float32) if cl_box is None else np.ascontiguousarray(cl_box, np.float32)


def imaging_core_nufft(u_dx, v_dy, vis_r, vis_i, vis_std, nx, ny, maxiter, eps, lambda_l1,
                       lambda_tv, lambda_tsv, cinit, xinit=None, nonneg_flag=1, box_flag=0,
                       cl_box=None, xout=None):
    u, v, vr, vi, vs = (_d(a) for a in (u_dx, v_dy, vis_r, vis_i, vis_std))
    n = nx * ny
    xi = np.zeros(n) if xinit is None else _d(xinit)
    xo = np.zeros(n) if xout is None else np.array(xout, np.float64, copy=True)
    box = _box(n, cl_box)
    res = RESULT()
    mfista_imaging_core_nufft(u, v, vr, vi, vs, u.size, nx, ny, maxiter, eps, lambda_l1, lambda_tv,
                              lambda_tsv, cinit, xi, xo, nonneg_flag, box_flag, box, res)
    _check()
    return xo, res.as_dict()


def imaging_core_fft(u_idx, v_idx, y_r, y_i, noise, nx, ny, maxiter, eps, lambda_l1, lambda_tv,
                     lambda_tsv, cinit, xinit=None, nonneg_flag=1, box_flag=0, cl_box=None,
                     xout=None):
    ui = np.ascontiguousarray(u_idx, np.int32)
    vi_ = np.ascontiguousarray(v_idx, np.int32)
    yr, yi, ns = (_d(a) for a in (y_r, y_i, noise))
    n = nx * ny
    xi = np.zeros(n) if xinit is None else _d(xinit)
    xo = np.zeros(n) if xout is None else np.array(xout, np.float64, copy=True)
    box = _box(n, cl_box)
    res = RESULT()
    mfista_imaging_core_fft(ui, vi_, yr, yi, ns, ui.size, nx, ny, maxiter, eps, lambda_l1, lambda_tv,
                            lambda_tsv, cinit, xi, xo, nonneg_flag, 64, box_flag, box, res)
    _check()
    return xo, res.as_dict()


def imaging_core_dft(y, A, nx, ny, maxiter, eps, lambda_l1, lambda_tv, lambda_tsv, cinit,
                     xinit=None, nonneg_flag=1, box_flag=0, cl_box=None):
    """A: logical (M, N) matrix; passed column-major as the reference expects."""
    A = np.asarray(A, np.float64)
    m, n = A.shape
    Af = np.asfortranarray(A)
    yy = _d(y)
    xi = np.zeros(n) if xinit is None else _d(xinit)
    xo = np.zeros(n)
    box = _box(n, cl_box)
    res = RESULT()
    mm, nn = C.c_int(m), C.c_int(n)
    lib().mfista_imaging_core_dft(_p(yy), Af.ctypes.data_as(_dp), C.byref(mm), C.byref(nn), nx, ny,
                                  maxiter, eps, lambda_l1, lambda_tv, lambda_tsv, cinit, _p(xi),
                                  _p(xo), nonneg_flag, 0, box_flag, _p(box, _fp), C.byref(res))
    _check()
    d = res.as_dict()
    if bool(res.residual):
        d["residual"] = np.ctypeslib.as_array(res.residual, shape=(m,)).copy()
        C.CDLL(None).free(C.cast(res.residual, C.c_void_p))
    return xo, d


def _problems(problems):
    arr = (Problem * len(problems))()
    for i, p in enumerate(problems):
        arr[i] = Problem(p["lambda_l1"], p.get("lambda_tv", 0.0), p.get("lambda_tsv", 0.0),
                         p["cinit"], p["maxiter"], p.get("nonneg_flag", 1),
                         p.get("target_cost", 0.0))
    return arr


def nufft_batch(u_dx, v_dy, vis_r, vis_i, vis_std, nx, ny, problems, eps, precision=FP64,
                pt_off=None, xinit=None, fgp_iter=100):
    """Solves len(problems) NUFFT problems in one batched GPU solve.

    problems: list of dicts with lambda_l1, lambda_tv, lambda_tsv, cinit,
    maxiter, nonneg_flag.  pt_off=None means every problem uses all points."""
    u, v, vr, vi, vs = (_d(a) for a in (u_dx, v_dy, vis_r, vis_i, vis_std))
    B = len(problems)
    shared = pt_off is None
    off = None if shared else np.ascontiguousarray(pt_off, np.int32)
    M = u.size if shared else 0
    n = nx * ny
    xi = None if xinit is None else _d(xinit)
    xo = np.zeros(B * n)
    res = (RESULT * B)()
    st = lib().mfista_nufft_batch(_p(u), _p(v), _p(vr), _p(vi), _p(vs), _p(off, _ip), int(shared), M,
                                  nx, ny, B, _problems(problems), eps, precision, fgp_iter, _p(xi),
                                  _p(xo), res)
    _check(st)
    return xo.reshape(B, n), [r.as_dict() for r in res]


def fft_batch(u_idx, v_idx, y_r, y_i, noise, nx, ny, problems, eps, precision=FP64, xinit=None,
              fgp_iter=100):
    """Solves len(problems) FFT-variant problems sharing one gridded data
    set (mfista_fft_batch); precision FP64 or FP32 (FP32 FFTs and FGP
    stencils with an FP64-corrected forward spectrum)."""
    ui = np.ascontiguousarray(u_idx, np.int32)
    vi_ = np.ascontiguousarray(v_idx, np.int32)
    yr, yi, ns = (_d(a) for a in (y_r, y_i, noise))
    B = len(problems)
    n = nx * ny
    xi = None if xinit is None else _d(xinit)
    xo = np.zeros(B * n)
    res = (RESULT * B)()
    st = lib().mfista_fft_batch(_p(ui, _ip), _p(vi_, _ip), _p(yr), _p(yi), _p(ns), ui.size, nx, ny, B,
                                _problems(problems), eps, precision, fgp_iter, _p(xi), _p(xo), res)
    _check(st)
    return xo.reshape(B, n), [r.as_dict() for r in res]


def fgp_profile(nx, ny, B, iters, precision=FP64, reps=10):
    """(ms per launch, compulsory bytes per launch) of the FGP TV prox for B
    problems of nx x ny with `iters` FGP iterations (mfista_fgp_profile)."""
    ms, by = C.c_double(), C.c_double()
    _check(lib().mfista_fgp_profile(nx, ny, B, iters, precision, reps, C.byref(ms), C.byref(by)))
    return ms.value, by.value


def dft_batch(y, A, nx, ny, problems, eps, xinit=None, fgp_iter=100, precision=None):
    """Solves len(problems) DFT problems sharing A (logical (M, N)) and y;
    precision FP64 (default) or BF16X3 (tensor-core split-BF16 GEMMs with
    FP64 anchor correction)."""
    precision = FP64 if precision is None else precision
    A = np.asarray(A, np.float64)
    m, n = A.shape
    Af = np.asfortranarray(A)
    yy = _d(y)
    B = len(problems)
    xi = None if xinit is None else _d(xinit)
    xo = np.zeros(B * n)
    res = (RESULT * B)()
    st = lib().mfista_dft_batch(_p(yy), Af.ctypes.data_as(_dp), m, n, nx, ny, B, _problems(problems), eps,
                                precision, fgp_iter, _p(xi), _p(xo), res)
    _check(st)
    return xo.reshape(B, n), [r.as_dict() for r in res]


def dft_apply(A, X, transpose=False, precision=None):
    """A @ x_b (or A.T @ x_b) for every row x_b of X, on the GPU; A is (M, N).
    precision FP64 or BF16X3 (the tensor-core split-BF16 GEMM alone)."""
    precision = FP64 if precision is None else precision
    A = np.asarray(A, np.float64)
    m, n = A.shape
    Af = np.asfortranarray(A)
    X = np.ascontiguousarray(np.atleast_2d(X), np.float64)
    B = X.shape[0]
    if X.shape[1] != (m if transpose else n):
        raise ValueError("X has the wrong length for this product")
    out = np.zeros((B, n if transpose else m))
    _check(lib().mfista_dft_apply(Af.ctypes.data_as(_dp), m, n, _p(X), B, int(bool(transpose)), precision,
                                  _p(out)))
    return out


def dft_profile(A, B, kernel, precision=None, reps=20):
    """(ms per launch, algorithmic bytes per launch) of the batched DFT GEMM
    `kernel` (0: A z, 1: A^T r) for B problems sharing A (M, N)."""
    precision = FP64 if precision is None else precision
    A = np.asarray(A, np.float64)
    m, n = A.shape
    Af = np.asfortranarray(A)
    ms, by = C.c_double(0), C.c_double(0)
    _check(lib().mfista_dft_profile(Af.ctypes.data_as(_dp), m, n, B, precision, kernel, reps, C.byref(ms),
                                    C.byref(by)))
    return ms.value, by.value


def nufft_movie(u_dx, v_dy, vis_r, vis_i, vis_std, pt_off, nx, ny, lambda_l1, lambda_tsv, lambda_t, cinit,
                maxiter, eps, nonneg_flag=1, t_list=None, xinit=None, c_box=None, precision=FP64):
    """Movie of len(pt_off) - 1 frames solved as one problem with the
    temporal term lambda_t sum_b |x_b - x_{b+1}|^2 / (t_{b+1} - t_b)
    (mfista_nufft_movie).  c_box: [nx*ny] pixel weights applied to the
    starting image and to every thresholded image (the matlab code's c_box).
    precision: FP64 or FP32 (corrected FP32 NUFFTs).  Returns (X [T][nx*ny],
    per-frame RESULT dicts, temporal cost at X)."""
    u, v, vr, vi, vs = (_d(a) for a in (u_dx, v_dy, vis_r, vis_i, vis_std))
    off = np.ascontiguousarray(pt_off, np.int32)
    T = off.size - 1
    xo = np.zeros(T * nx * ny)
    res = (RESULT * T)()
    tc = C.c_double(0)
    tl = None if t_list is None else _d(t_list)
    xi = None if xinit is None else _d(xinit)
    cb = None if c_box is None else _d(c_box)
    if cb is not None and cb.size != nx * ny:
        raise ValueError("c_box needs nx * ny values")
    _check(lib().mfista_nufft_movie(_p(u), _p(v), _p(vr), _p(vi), _p(vs), off.ctypes.data_as(_ip), T, nx, ny,
                                    _p(tl), lambda_l1, lambda_tsv, lambda_t, cinit, maxiter, eps, nonneg_flag,
                                    _p(cb), precision, _p(xi), _p(xo), res, C.byref(tc)))
    return xo.reshape(T, nx * ny), [r.as_dict() for r in res], tc.value


def cpp_x2y_nufft(u_dx, v_dy, nx, ny, x):
    """Forward NUFFT of the reference's C++ build (x2y_nufft: 12-tap
    kernel, floor binning) on the GPU; returns (real, imag)."""
    u, v, xx = _d(u_dx), _d(v_dy), _d(x)
    yr, yi = np.zeros(u.size), np.zeros(u.size)
    _check(lib().mfista_cpp_x2y_nufft(_p(u), _p(v), u.size, nx, ny, _p(xx), _p(yr), _p(yi)))
    return yr, yi


def cpp_y2x_nufft(u_dx, v_dy, nx, ny, y_r, y_i):
    """Adjoint NUFFT of the reference's C++ build (y2x_nufft) on the GPU."""
    u, v, yr, yi = (_d(a) for a in (u_dx, v_dy, y_r, y_i))
    x = np.zeros(nx * ny)
    _check(lib().mfista_cpp_y2x_nufft(_p(u), _p(v), u.size, nx, ny, _p(yr), _p(yi), _p(x)))
    return x


def cpp_imaging_core_nufft(u_dx, v_dy, vis_r, vis_i, vis_std, nx, ny, maxiter, eps, lambda_l1, lambda_tv,
                           lambda_tsv, cinit, xinit=None, nonneg_flag=1, box_flag=0, cl_box=None, xout=None):
    """The C++ build's mfista_imaging_core_nufft.  Like it, the call sorts
    the five point arrays in place: pass float64 contiguous arrays to see
    the permutation (other inputs are converted, and the copies sorted)."""
    u, v, vr, vi, vs = (a if isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous
                        else _d(a) for a in (u_dx, v_dy, vis_r, vis_i, vis_std))
    n = nx * ny
    xi = np.zeros(n) if xinit is None else _d(xinit)
    xo = np.zeros(n) if xout is None else np.array(xout, np.float64, copy=True)
    box = _box(n, cl_box)
    res = RESULT()
    lib().mfista_cpp_imaging_core_nufft(_p(u), _p(v), _p(vr), _p(vi), _p(vs), u.size, nx, ny, maxiter, eps,
                                        lambda_l1, lambda_tv, lambda_tsv, cinit, _p(xi), _p(xo), nonneg_flag,
                                        box_flag, _p(box, _fp), C.byref(res))
    _check()
    return xo, res.as_dict()


def dft_looe(y, A, X, nx, lambda_tsv=None):
    """Approximate leave-one-out error of DFT solutions (the reference's
    c/looe_lib.c) on the GPU: A is (M, N), X the solutions [B][N] (e.g. a
    lambda grid's from dft_batch), lambda_tsv None (L1 form) or per
    solution.  Returns (looe_m [B], looe_std [B], hessian_positive [B])."""
    A = np.asarray(A, np.float64)
    m, n = A.shape
    Af = np.asfortranarray(A)
    X = np.ascontiguousarray(np.atleast_2d(X), np.float64)
    B = X.shape[0]
    lt = None if lambda_tsv is None else _d(np.broadcast_to(np.asarray(lambda_tsv, np.float64), (B,)))
    om, osd = np.zeros(B), np.zeros(B)
    pos = np.zeros(B, np.int32)
    _check(lib().mfista_dft_looe(_p(_d(y)), Af.ctypes.data_as(_dp), m, n, nx, _p(X), B, _p(lt), _p(om), _p(osd),
                                 pos.ctypes.data_as(_ip)))
    return om, osd, pos.astype(bool)


class Plan:
    """Device-resident batched NUFFT plan (geometry uploaded once)."""

    def __init__(self, u_dx, v_dy, vis_r, vis_i, vis_std, nx, ny, B, precision=FP64, pt_off=None,
                 form_tv=False, fgp_iter=100):
        self._keep = [_d(a) for a in (u_dx, v_dy, vis_r, vis_i, vis_std)]
        u, v, vr, vi, vs = self._keep
        shared = pt_off is None
        off = None if shared else np.ascontiguousarray(pt_off, np.int32)
        self.B, self.n = B, nx * ny
        h = lib().mfista_nufft_plan_create(_p(u), _p(v), _p(vr), _p(vi), _p(vs), _p(off, _ip),
                                           int(shared), u.size if shared else 0, nx, ny, B,
                                           precision, int(form_tv), fgp_iter)
        if not h:
            _check()
        self.h = h

    def set_problems(self, problems, eps, xinit=None):
        self._probs = _problems(problems)
        self._xi = None if xinit is None else _d(xinit)
        _check(lib().mfista_plan_set_problems(self.h, self._probs, eps, _p(self._xi)))

    def run(self):
        _check(lib().mfista_plan_run(self.h))

    def fetch(self, want_x=True, check=True):
        """(xout [B, N] or None, RESULT dicts).  check=False returns the
        results of problems that stopped with a status instead of raising;
        each dict then carries its own 'status'."""
        xo = np.zeros(self.B * self.n) if want_x else None
        res = (RESULT * self.B)()
        st = lib().mfista_plan_fetch(self.h, _p(xo), res)
        if check:
            _check(st)
        out = [r.as_dict() for r in res]
        if not check:
            stat = (C.c_int * self.B)()
            lib().mfista_plan_statuses(self.h, stat)
            for d, s in zip(out, stat):
                d["status"] = int(s)
        return (None if xo is None else xo.reshape(self.B, self.n)), out

    def profile(self, kernel, reps=20):
        """(ms per launch, algorithmic bytes per launch) of one operator kernel."""
        ms, by = C.c_double(0), C.c_double(0)
        _check(lib().mfista_plan_profile(self.h, kernel, reps, C.byref(ms), C.byref(by)))
        return ms.value, by.value

    SHAPE_KEYS = ("interp_ppw", "spread_cluster", "rows_per_cta", "cols_per_cta")

    def shapes(self):
        """Launch shapes of the operator kernels (0 = not used by this plan)."""
        a = (C.c_int * 4)()
        _check(lib().mfista_plan_get_shapes(self.h, a))
        return dict(zip(self.SHAPE_KEYS, list(a)))

    def set_shapes(self, **shapes):
        """Sets some launch shapes (the others keep their value) and captures
        the solve graph again."""
        unknown = set(shapes) - set(self.SHAPE_KEYS)
        if unknown:
            raise ValueError(f"unknown shape keys {sorted(unknown)}")
        a = (C.c_int * 4)(*[int(shapes.get(k, 0)) for k in self.SHAPE_KEYS])
        _check(lib().mfista_plan_set_shapes(self.h, a))

    def tune(self, reps=10):
        """Autotunes the launch shapes on this GPU (scoring each candidate
        on the whole batch and on one active problem); returns (shapes, ms
        per launch of each knob's kernels at the chosen shape, whole batch
        active).  Iterates are left undefined: call set_problems before the
        next run."""
        a = (C.c_int * 4)()
        ms = np.zeros(4)
        _check(lib().mfista_plan_tune(self.h, reps, a, _p(ms)))
        return dict(zip(self.SHAPE_KEYS, list(a))), dict(zip(self.SHAPE_KEYS, ms.tolist()))

    @property
    def stream(self):
        return lib().mfista_plan_stream(self.h)

    @property
    def device_loop(self):
        return bool(lib().mfista_plan_device_loop(self.h))

    @property
    def kernel_launches(self):
        return lib().mfista_plan_kernel_launches(self.h)

    def close(self):
        if getattr(self, "h", None):
            lib().mfista_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def nufft_forward(u_dx, v_dy, nx, ny, x, precision=FP64):
    u, v, xx = _d(u_dx), _d(v_dy), _d(x)
    fr = np.zeros(u.size)
    fi = np.zeros(u.size)
    _check(lib().mfista_nufft_forward(_p(u), _p(v), u.size, nx, ny, _p(xx), _p(fr), _p(fi), precision))
    return fr, fi


def nufft_adjoint(u_dx, v_dy, nx, ny, r_r, r_i, precision=FP64):
    u, v, a, b = _d(u_dx), _d(v_dy), _d(r_r), _d(r_i)
    out = np.zeros(nx * ny)
    _check(lib().mfista_nufft_adjoint(_p(u), _p(v), u.size, nx, ny, _p(a), _p(b), _p(out), precision))
    return out


def fgp_prox(b, nx, ny, lambda_l1, lambda_tv, iters, nonneg_flag, cl_box=None, precision=FP64):
    bb = _d(b)
    out = np.zeros(nx * ny)
    box = None if cl_box is None else np.ascontiguousarray(cl_box, np.float32)
    _check(lib().mfista_fgp_prox(_p(bb), nx, ny, lambda_l1, lambda_tv, iters, nonneg_flag,
                                 0 if box is None else 1, _p(box, _fp), _p(out), precision))
    return out


def nufft_lipschitz(u_dx, v_dy, vis_std, nx, ny, iters=30):
    u, v, s = _d(u_dx), _d(v_dy), _d(vis_std)
    out = C.c_double(0.0)
    _check(lib().mfista_nufft_lipschitz(_p(u), _p(v), _p(s), u.size, nx, ny, iters, C.byref(out)))
    return out.value
