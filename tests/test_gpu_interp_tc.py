"""Tensor-core interpolation and spreading (FP32 form, k_nufft_interp_tc,
k_nufft_spread_tc) against the CUDA-core FP32 kernels and the FP64 operator.

The tensor-core kernel stages each tile's 32 x 32 window of virtual cells
(wrapped rows, Hermitian-mirrored columns with the conjugate, dropped taps
as zeros) and takes the separable tap sums as 3-pass TF32 products, so it
must agree with the per-tap FP32 kernel to FP32 rounding (2e-6 relative L2)
and with FP64 as every FP32 operator does (2e-5).  The geometries cover
the lambda-grid workload, non-power-of-two grids, points near the Nyquist
edges (taps dropped or mirrored) and points on the v = 0 fold.  The
tensor-core spreading sums every stored cell over the "virtual points"
(each point direct and mirrored) listed for its 8 x 16 tile, long lists in
segments added by the last CTA of the tile: the same bounds.
"""
import os

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


def _with_env(name, on, fn):
    old = os.environ.get(name)
    os.environ[name] = "1" if on else "0"
    try:
        return fn()
    finally:
        if old is None:
            del os.environ[name]
        else:
            os.environ[name] = old


def _forward(gpulib, u, v, nx, x, tc):
    fr, fi = _with_env("MFISTA_INTERP_TC", tc, lambda: gpulib.nufft_forward(u, v, nx, nx, x, precision=gpulib.FP32))
    return fr + 1j * fi


def _adjoint(gpulib, u, v, nx, a, b, tc):
    return _with_env("MFISTA_SPREAD_TC", tc,
                     lambda: gpulib.nufft_adjoint(u, v, nx, nx, a, b, precision=gpulib.FP32))


def _geometries():
    from sparseimaging_b200 import synth
    out = []
    p = synth.lambda_grid_problem()
    out.append(("lambda_grid_128", p.u_dx, p.v_dy, p.nx))
    for nx, kfrac in [(200, 1.0), (96, 0.5), (64, 1.0)]:
        rng = np.random.default_rng(nx)
        u, v = synth.earth_rotation_uv(7, 40, seed=None, rng=rng)
        u_dx, v_dy = synth.scale_uv_to_radians(u, v, nx, max(1, int(synth.safe_kmax(nx) * kfrac)))
        out.append((f"earth_rotation_{nx}", u_dx, v_dy, nx))
    nx = 32
    rng = np.random.default_rng(5)
    edge = np.array([15.5, -15.9, 15.99, -16.0, 0.0, 0.4, -0.4, 7.3, -11.2])
    u = 2 * np.pi * np.concatenate([edge, rng.uniform(-16, 16, 200)]) / (2 * nx)
    v = 2 * np.pi * np.concatenate([edge[::-1], rng.uniform(-16, 16, 200)]) / (2 * nx)
    out.append(("nyquist_edges_32", u * 2, v * 2, nx))
    v0 = np.zeros(50)
    out.append(("fold_v0_48", rng.uniform(-np.pi, np.pi, 50), v0, 48))
    return out


@pytest.mark.parametrize("case", range(6))
def test_tensor_core_interpolation_matches(gpulib, case):
    name, u, v, nx = _geometries()[case]
    x = np.random.default_rng(case).random(nx * nx)
    tc = _forward(gpulib, u, v, nx, x, True)
    cc = _forward(gpulib, u, v, nx, x, False)
    fr, fi = gpulib.nufft_forward(u, v, nx, nx, x)
    f64 = fr + 1j * fi
    assert rel(tc, cc) < 2e-6, name
    assert rel(tc, f64) < 2e-5, name


@pytest.mark.parametrize("case", range(6))
def test_tensor_core_spreading_matches(gpulib, case):
    name, u, v, nx = _geometries()[case]
    rng = np.random.default_rng(100 + case)
    a, b = rng.standard_normal(u.size), rng.standard_normal(u.size)
    tc = _adjoint(gpulib, u, v, nx, a, b, True)
    cc = _adjoint(gpulib, u, v, nx, a, b, False)
    f64 = gpulib.nufft_adjoint(u, v, nx, nx, a, b)
    assert rel(tc, cc) < 2e-6, name
    assert rel(tc, f64) < 2e-5, name
