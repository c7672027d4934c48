"""Tensor-core interpolation (FP32 form, k_nufft_interp_tc) against the
CUDA-core FP32 kernel and the FP64 operator.

The tensor-core kernel stages each tile's 32 x 32 window of virtual cells
(wrapped rows, Hermitian-mirrored columns with the conjugate, dropped taps
as zeros) and takes the separable tap sums as 3-pass TF32 products, so it
must agree with the per-tap FP32 kernel to FP32 rounding (2e-6 relative L2)
and with FP64 as every FP32 operator does (2e-5).  The geometries cover
the lambda-grid workload, non-power-of-two grids, points near the Nyquist
edges (taps dropped or mirrored) and points on the v = 0 fold.
"""
import os

import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


def _forward(gpulib, u, v, nx, x, tc):
    old = os.environ.get("MFISTA_INTERP_TC")
    os.environ["MFISTA_INTERP_TC"] = "1" if tc else "0"
    try:
        fr, fi = gpulib.nufft_forward(u, v, nx, nx, x, precision=gpulib.FP32)
    finally:
        if old is None:
            del os.environ["MFISTA_INTERP_TC"]
        else:
            os.environ["MFISTA_INTERP_TC"] = old
    return fr + 1j * fi


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
