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
