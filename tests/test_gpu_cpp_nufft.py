"""Forward NUFFT of the reference's C++ build on the GPU
(mfista_cpp_x2y_nufft) against its restatement (oracle/cpp_nufft_oracle.py,
itself pinned by the exact DFT and adjointness) and the exact DFT."""
import numpy as np
import pytest

from conftest import rel
from oracle.cpp_nufft_oracle import CppNufftPlan

pytestmark = pytest.mark.gpu


def test_cpp_forward_matches_oracle_and_dft(gpulib, c0):
    from sparseimaging_b200 import synth
    sky = c0["sky"].reshape(64, 64)
    gr, gi = gpulib.cpp_x2y_nufft(c0["u"], c0["v"], 64, 64, sky.ravel())
    orr, ori = CppNufftPlan(c0["u"], c0["v"], 64, 64).forward(sky.ravel())
    assert rel(gr + 1j * gi, orr + 1j * ori) < 1e-12
    assert rel(gr + 1j * gi, synth.dft_vis(sky, c0["u"], c0["v"])) < 1e-6
    rng = np.random.default_rng(3)
    x = rng.standard_normal(64 * 64)
    gr, gi = gpulib.cpp_x2y_nufft(c0["u"], c0["v"], 64, 64, x)
    orr, ori = CppNufftPlan(c0["u"], c0["v"], 64, 64).forward(x)
    assert rel(gr + 1j * gi, orr + 1j * ori) < 1e-12


def test_cpp_forward_rejects_small_grids(gpulib, c0):
    with pytest.raises(gpulib.MfistaError):
        gpulib.cpp_x2y_nufft(c0["u"], c0["v"], 8, 8, np.zeros(64))


def test_cpp_adjoint_matches_oracle_and_is_the_adjoint(gpulib, c0):
    """y2x_nufft on the GPU (gather over the Hermitian halo folds) against
    the restatement of NUFFT2d1_sngl, and <A x, y> = <x, A^H y> with the
    GPU's own forward."""
    rng = np.random.default_rng(8)
    m = c0["u"].size
    a, b = rng.standard_normal(m), rng.standard_normal(m)
    got = gpulib.cpp_y2x_nufft(c0["u"], c0["v"], 64, 64, a, b)
    want = CppNufftPlan(c0["u"], c0["v"], 64, 64).adjoint(a, b)
    assert rel(got, want) < 1e-12
    x = rng.standard_normal(64 * 64)
    fr, fi = gpulib.cpp_x2y_nufft(c0["u"], c0["v"], 64, 64, x)
    lhs = fr @ a + fi @ b
    assert abs(lhs - x @ got) <= 1e-11 * abs(lhs)


def test_cpp_adjoint_near_nyquist_and_edges(gpulib):
    """Points whose 12-tap blocks cross ky = 0, ky = Ny and kx = -Nx (every
    halo fold) on a rectangular grid."""
    rng = np.random.default_rng(9)
    nx, ny, m = 32, 24, 400
    kmax = 2 * np.pi * (nx - 7) / (2 * nx)
    u = rng.uniform(-kmax, kmax, m)
    v = rng.uniform(-kmax, kmax, m)
    v[:40] = rng.uniform(-0.05, 0.05, 40)          # near ky = 0
    u[40:80] = -np.pi * (1 - 1e-3)                  # near kx = -Nx
    a, b = rng.standard_normal(m), rng.standard_normal(m)
    got = gpulib.cpp_y2x_nufft(u, v, nx, ny, a, b)
    want = CppNufftPlan(u, v, nx, ny).adjoint(a, b)
    assert rel(got, want) < 1e-12


def _cpp_objective(c0, x, lam, lts):
    from oracle import mfista_oracle as R
    P = CppNufftPlan(c0["u"], c0["v"], 64, 64)
    fr, fi = P.forward(x)
    w = 1.0 / c0["vis_std"]
    rr, ri = (c0["vis_r"] - fr) * w, (c0["vis_i"] - fi) * w
    chisq = rr @ rr + ri @ ri
    return chisq, chisq / 2 + lam * np.abs(x).sum() + lts * R.tsv(64, 64, x)


def _arrays(c0):
    return [np.array(c0[k], np.float64) for k in ("u", "v", "vis_r", "vis_i", "vis_std")]


def test_cpp_solver_matches_cpp_loop_oracle(gpulib, c0):
    """The C++ build's mfista_imaging_core_nufft on the GPU against the
    restated C++ loop (its operators, first backtracking factor 10), 100
    iterations of config 0; RESULT as calc_costs_nufft fills it (M = M)."""
    from oracle.cpp_nufft_oracle import cpp_imaging_core_nufft
    lam, lip = float(c0["lam1"]), float(c0["cinit"])
    lts = 1e-3 * lam
    x, r = gpulib.cpp_imaging_core_nufft(*_arrays(c0), 64, 64, 100, 1e-5, lam, 0.0, lts, lip)
    xo, it, c = cpp_imaging_core_nufft(c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"], 64, 64, 100,
                                       1e-5, lam, lts, lip, np.zeros(64 * 64), 1)
    assert r["ITER"] == it == 100
    assert rel(x, xo) < 1e-8
    assert abs(r["Lip_const"] - c) <= 1e-12 * c
    chisq, f = _cpp_objective(c0, xo, lam, lts)
    assert r["M"] == c0["u"].size
    assert abs(r["sq_error"] - chisq) <= 1e-9 * chisq
    assert abs(r["finalcost"] - f) <= 1e-9 * f
    assert abs(r["mean_sq_error"] - chisq / c0["u"].size) <= 1e-9 * chisq / c0["u"].size


def test_cpp_first_iteration_backtracks_by_ten(gpulib, c0):
    """From a step size far too small, the first iteration of the C++ loop
    multiplies c by 10 per failed trial, then divides by 1.1 once: the GPU
    solve's c after one iteration is cinit 10^k / 1.1 with the oracle's k."""
    from oracle.cpp_nufft_oracle import cpp_imaging_core_nufft
    lam, lip = float(c0["lam1"]), float(c0["cinit"])
    cinit = lip * 1e-6
    _, r = gpulib.cpp_imaging_core_nufft(*_arrays(c0), 64, 64, 1, 1e-5, lam, 0.0, 1e-3 * lam, cinit)
    _, it, c = cpp_imaging_core_nufft(c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"], 64, 64, 1, 1e-5,
                                      lam, 1e-3 * lam, cinit, np.zeros(64 * 64), 1)
    k = np.log10(r["Lip_const"] * 1.1 / cinit)
    assert k > 0.5 and abs(k - round(k)) < 1e-9
    assert abs(r["Lip_const"] - c) <= 1e-12 * c


def test_cpp_solver_sorts_caller_arrays(gpulib, c0):
    """sort_input: the caller's five arrays come back permuted into grid
    order of v, then u (c++/mfista_nufft_lib.cpp:550-641)."""
    arrs = _arrays(c0)
    orig = [a.copy() for a in arrs]
    lam, lip = float(c0["lam1"]), float(c0["cinit"])
    gpulib.cpp_imaging_core_nufft(*arrs, 64, 64, 5, 1e-5, lam, 0.0, 1e-3 * lam, lip)
    kv = np.round(arrs[1] * 128 / (2 * np.pi))
    ku = np.round(arrs[0] * 128 / (2 * np.pi))
    keys = list(zip(kv, ku))
    assert keys == sorted(keys)
    # a permutation of the rows (all five arrays moved together)
    assert sorted(zip(*[a.tolist() for a in orig])) == sorted(zip(*[a.tolist() for a in arrs]))


def test_cpp_solver_has_no_tv_form(gpulib, c0):
    lam, lip = float(c0["lam1"]), float(c0["cinit"])
    with pytest.raises(gpulib.MfistaError):
        gpulib.cpp_imaging_core_nufft(*_arrays(c0), 64, 64, 5, 1e-5, lam, 1e-3 * lam, 0.0, lip)


def test_cpp_build_library_exports_forward_to_gpu(gpulib, c0):
    """libmfista_b200_cpp.so: the C++ build's own names (x2y_nufft,
    y2x_nufft, mfista_imaging_core_nufft) give the C++-build results."""
    import ctypes as C
    from sparseimaging_b200 import build
    L = C.CDLL(build.CPP_LIB)
    dp = C.POINTER(C.c_double)
    m = c0["u"].size
    u, v = np.array(c0["u"]), np.array(c0["v"])
    rng = np.random.default_rng(10)
    x = rng.standard_normal(64 * 64)
    yr, yi = np.zeros(m), np.zeros(m)
    L.x2y_nufft(u.ctypes.data_as(dp), v.ctypes.data_as(dp), m, 64, 64, x.ctypes.data_as(dp),
                yr.ctypes.data_as(dp), yi.ctypes.data_as(dp))
    wr, wi = CppNufftPlan(u, v, 64, 64).forward(x)
    assert rel(yr + 1j * yi, wr + 1j * wi) < 1e-12
    xo = np.zeros(64 * 64)
    L.y2x_nufft(u.ctypes.data_as(dp), v.ctypes.data_as(dp), m, 64, 64, yr.ctypes.data_as(dp),
                yi.ctypes.data_as(dp), xo.ctypes.data_as(dp))
    assert rel(xo, CppNufftPlan(u, v, 64, 64).adjoint(yr, yi)) < 1e-12
    # the solver name resolves to the C++ build's solver (M = M in RESULT)
    arrs = _arrays(c0)
    lam, lip = float(c0["lam1"]), float(c0["cinit"])
    res = gpulib.RESULT()
    xout, xinit = np.zeros(64 * 64), np.zeros(64 * 64)
    box = np.ones(64 * 64, np.float32)
    L.mfista_imaging_core_nufft(*[a.ctypes.data_as(dp) for a in arrs], C.c_int(m), C.c_int(64), C.c_int(64),
                                C.c_int(20), C.c_double(1e-5), C.c_double(lam), C.c_double(0.0),
                                C.c_double(1e-3 * lam), C.c_double(lip), xinit.ctypes.data_as(dp),
                                xout.ctypes.data_as(dp), C.c_int(1), C.c_int(0),
                                box.ctypes.data_as(C.POINTER(C.c_float)), C.byref(res))
    assert gpulib.last_status() == 0
    assert res.M == m and res.ITER == 20
    x2, r2 = gpulib.cpp_imaging_core_nufft(*_arrays(c0), 64, 64, 20, 1e-5, lam, 0.0, 1e-3 * lam, lip)
    assert np.array_equal(xout, x2)
