"""The restatement of the C++ build's NUFFT (oracle/cpp_nufft_oracle.py:
MSP = 6, floor binning, Hermitian halos).  The C++ sources need Eigen, which
is not in this image, so the restatement is pinned by what the operators
must be: the forward approximates the exact DFT that the C library's NUFFT
also approximates (to a 12-tap kernel's accuracy), the adjoint is its exact
adjoint, and it agrees with the C library's adjoint to that accuracy."""
import numpy as np

from conftest import rel
from oracle import mfista_oracle as R
from oracle.cpp_nufft_oracle import CppNufftPlan
from sparseimaging_b200 import synth


def test_forward_is_the_dft(c0):
    sky = c0["sky"].reshape(64, 64)
    fr, fi = CppNufftPlan(c0["u"], c0["v"], 64, 64).forward(sky.ravel())
    assert rel(fr + 1j * fi, synth.dft_vis(sky, c0["u"], c0["v"])) < 1e-6


def test_adjoint_is_the_exact_adjoint(c0):
    P = CppNufftPlan(c0["u"], c0["v"], 64, 64)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(64 * 64)
    a, b = rng.standard_normal(c0["u"].size), rng.standard_normal(c0["u"].size)
    fr, fi = P.forward(x)
    lhs = fr @ a + fi @ b
    assert abs(lhs - x @ P.adjoint(a, b)) <= 1e-12 * abs(lhs)


def test_adjoint_matches_the_c_library_adjoint(c0):
    rng = np.random.default_rng(6)
    a, b = rng.standard_normal(c0["u"].size), rng.standard_normal(c0["u"].size)
    got = CppNufftPlan(c0["u"], c0["v"], 64, 64).adjoint(a, b)
    want = R.NufftPlan(c0["u"], c0["v"], 64, 64).adjoint(a, b)
    assert rel(got, want) < 1e-5


def test_cpp_loop_lands_near_the_c_loop(c0):
    """The C++ build's loop (its operators, a backtracking factor of 10 in
    the first iteration) and the C library's reach nearly the same image:
    the operators differ by the 12-tap kernel's error."""
    from oracle.cpp_nufft_oracle import cpp_imaging_core_nufft
    lam, lip = float(c0["lam1"]), float(c0["cinit"])
    args = (c0["u"], c0["v"], c0["vis_r"], c0["vis_i"], c0["vis_std"], 64, 64, 100, 1e-5)
    x_c, _ = R.imaging_core_nufft(*args, lam, 0.0, 1e-3 * lam, lip, np.zeros(64 * 64), 1)
    x_p, it, _ = cpp_imaging_core_nufft(*args, lam, 1e-3 * lam, lip, np.zeros(64 * 64), 1)
    assert it == 100
    assert rel(x_p, x_c) < 1e-3


def test_first_backtracking_factor_is_ten(c0):
    """From a step size far too small, the first iteration multiplies c by
    10 per failed trial (then divides by 1.1 once) in the C++ loop, by 1.1
    in the C loop."""
    from oracle.cpp_nufft_oracle import CppNufftPlan
    lam, lip = float(c0["lam1"]), float(c0["cinit"])
    w = 1.0 / c0["vis_std"]
    for eta_first, base in ((10.0, 10.0), (None, 1.1)):
        P = CppNufftPlan(c0["u"], c0["v"], 64, 64)

        def f_part(x):
            fr, fi = P.forward(x)
            rr, ri = (c0["vis_r"] - fr) * w, (c0["vis_i"] - fi) * w
            return 0.5 * (rr @ rr + ri @ ri), (rr, ri)

        cinit = lip * 1e-6
        _, _, c = R.mfista(f_part, lambda r: P.adjoint(r[0] * w, r[1] * w), np.zeros(64 * 64), 64, 64, 1, 0.0,
                           lam, 0.0, 1e-3 * lam, cinit, 1, eta_first=eta_first)
        k = np.log(c * 1.1 / cinit) / np.log(base)
        assert k > 0.5 and abs(k - round(k)) < 1e-9
