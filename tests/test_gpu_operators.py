"""GPU operators against the reference's outputs and the oracle.

Tolerances: FP64 operators within 1e-12 relative L2 of the reference (the
FFT and the summation order differ, so bit equality is not expected);
FP32 operators within 2e-5 relative L2.
"""
import numpy as np
import pytest

from conftest import rel
from oracle import mfista_oracle as O

pytestmark = pytest.mark.gpu


def test_nufft_forward_fp64(gpulib, c0):
    fr, fi = gpulib.nufft_forward(c0["u"], c0["v"], 64, 64, c0["sky"])
    assert rel(fr + 1j * fi, c0["fwd_r"] + 1j * c0["fwd_i"]) < 1e-12


def test_nufft_adjoint_fp64(gpulib, c0):
    x = gpulib.nufft_adjoint(c0["u"], c0["v"], 64, 64, c0["adj_in_r"], c0["adj_in_i"])
    assert rel(x, c0["adj_out"]) < 1e-12


def test_nufft_fp32(gpulib, c0):
    fr, fi = gpulib.nufft_forward(c0["u"], c0["v"], 64, 64, c0["sky"], precision=gpulib.FP32)
    assert rel(fr + 1j * fi, c0["fwd_r"] + 1j * c0["fwd_i"]) < 2e-5
    x = gpulib.nufft_adjoint(c0["u"], c0["v"], 64, 64, c0["adj_in_r"], c0["adj_in_i"],
                             precision=gpulib.FP32)
    assert rel(x, c0["adj_out"]) < 2e-5


@pytest.mark.parametrize("nx,kfrac", [(128, 1.0), (200, 1.0), (96, 0.5), (256, 1.0)])
def test_nufft_sizes_vs_oracle(gpulib, nx, kfrac):
    """Other grid sizes, including non-powers of two (2Nx = 400, 192)."""
    from sparseimaging_b200 import synth
    rng = np.random.default_rng(nx)
    u, v = synth.earth_rotation_uv(7, 40, seed=None, rng=rng)
    u_dx, v_dy = synth.scale_uv_to_radians(u, v, nx, max(1, int(synth.safe_kmax(nx) * kfrac)))
    plan = O.NufftPlan(u_dx, v_dy, nx, nx)
    x = rng.random(nx * nx)
    fr, fi = gpulib.nufft_forward(u_dx, v_dy, nx, nx, x)
    gr, gi = plan.forward(x)
    assert rel(fr + 1j * fi, gr + 1j * gi) < 1e-12
    a, b = rng.standard_normal(u_dx.size), rng.standard_normal(u_dx.size)
    assert rel(gpulib.nufft_adjoint(u_dx, v_dy, nx, nx, a, b), plan.adjoint(a, b)) < 1e-12


def test_nufft_near_nyquist_drops_out_of_range_taps(gpulib):
    """Points whose footprint leaves [-Nx, Nx) (the reference indexes outside
    its grid there): taps outside are dropped, as the oracle does."""
    nx = 32
    u = np.array([2 * np.pi * 15.5 / nx, -2 * np.pi * 15.9 / nx, 0.1])
    v = np.array([2 * np.pi * 15.7 / nx, 2 * np.pi * -15.9 / nx, -0.2])
    plan = O.NufftPlan(u, v, nx, nx)
    x = np.random.default_rng(1).random(nx * nx)
    fr, fi = gpulib.nufft_forward(u, v, nx, nx, x)
    gr, gi = plan.forward(x)
    assert rel(fr + 1j * fi, gr + 1j * gi) < 1e-12
    a, b = np.ones(3), np.arange(3.0)
    assert rel(gpulib.nufft_adjoint(u, v, nx, nx, a, b), plan.adjoint(a, b)) < 1e-12


def test_nufft_adjointness_fp64(gpulib, c0):
    rng = np.random.default_rng(9)
    x = rng.standard_normal(64 * 64)
    a, b = rng.standard_normal(c0["u"].size), rng.standard_normal(c0["u"].size)
    fr, fi = gpulib.nufft_forward(c0["u"], c0["v"], 64, 64, x)
    y = gpulib.nufft_adjoint(c0["u"], c0["v"], 64, 64, a, b)
    assert abs((fr @ a + fi @ b) - x @ y) <= 1e-11 * abs(x @ y)


def test_fgp_prox_fp64(gpulib, c1):
    b = c1["fgp_b"]
    assert rel(gpulib.fgp_prox(b, 128, 128, 0.0, 2e-4, 100, 1), c1["fgp_nonneg"]) < 1e-12
    assert rel(gpulib.fgp_prox(b, 128, 128, 1e-5, 2e-4, 100, 0), c1["fgp_l1"]) < 1e-12


def test_fgp_prox_fp32(gpulib, c1):
    b = c1["fgp_b"]
    assert rel(gpulib.fgp_prox(b, 128, 128, 0.0, 2e-4, 100, 1, precision=gpulib.FP32),
               c1["fgp_nonneg"]) < 1e-5


@pytest.mark.parametrize("nx,ny", [(64, 48), (256, 256), (300, 17), (1024, 600)])
def test_fgp_prox_shapes_vs_oracle(gpulib, nx, ny):
    """Cluster slabs with uneven rows (300 x 17), 16-CTA clusters (256^2) and
    the global-memory slabs (1024 x 600)."""
    rng = np.random.default_rng(nx + ny)
    b = rng.random(nx * ny)
    box = (rng.random(nx * ny) > 0.1).astype(np.float32)
    for nonneg in (0, 1):
        got = gpulib.fgp_prox(b, nx, ny, 0.05, 0.02, 20, nonneg, cl_box=box)
        want = O.fgp(nx, ny, b, 0.0 if nonneg else 0.05, 0.02, 20, bool(nonneg), box)
        assert rel(got, want) < 1e-12


def test_lipschitz_estimate(gpulib, c0):
    lip = gpulib.nufft_lipschitz(c0["u"], c0["v"], c0["vis_std"], 64, 64, iters=30)
    assert abs(lip - float(c0["cinit"])) <= 1e-3 * float(c0["cinit"])
