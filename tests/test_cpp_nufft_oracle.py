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
