"""The matrix forms behind the tensor-core NUFFT kernels, checked in numpy
against the per-tap rules of the CUDA-core kernels (no GPU).

Interpolation (k_nufft_interp_tc): a point's value is its 24 x 24 taps over
the stored half grid (rows wrapped, columns beyond the half plane mirrored
with the conjugate, taps outside dropped, the imaginary part of direct taps
negated).  The kernel instead resolves every *virtual* cell of a 32 x 32
window once (stored cell, sign of the imaginary part, or zero) and sums
separable weights over the window: the same numbers.

Spreading (k_nufft_spread_tc): a stored cell sums, over the points, half
the residual times the weights of the point's direct taps on it (imaginary
part negated) and of its mirrored taps (imaginary part kept).  The kernel
lists "virtual points" per 8 x 16 tile -- every point direct, and mirrored
with first tap (-mx - 12, -my - 12) and reversed weight vectors -- and sums
them with the direct rule only: the same numbers."""
import numpy as np

MSP, TAPS = 12, 24


def wrap_row(m, nx):
    if 0 <= m < nx:
        return m
    if -nx <= m < 0:
        return m + 2 * nx
    return -1


def half_col(m, ny):
    if 0 <= m < ny:
        return m
    if m == -ny:
        return ny
    return -1


def _case(nx, M, seed):
    rng = np.random.default_rng(seed)
    mx = rng.integers(-nx, nx + 1, M)
    my = rng.integers(-nx, nx + 1, M)
    mx[:4] = [nx, -nx, 0, 3]
    my[:4] = [nx, -nx, 0, -1]
    wx, wy = rng.random((M, TAPS)), rng.random((M, TAPS))
    return mx, my, wx, wy, rng


def test_interpolation_window_equals_per_tap_rule():
    nx = ny = 16
    mx, my, wx, wy, rng = _case(nx, 40, 1)
    grid = rng.standard_normal((2 * nx, ny + 1)) + 1j * rng.standard_normal((2 * nx, ny + 1))
    for k in range(len(mx)):
        # per-tap rule of the CUDA-core kernels
        ref = 0j
        for lx in range(TAPS):
            for ly in range(TAPS):
                m, mxm = my[k] + ly - (MSP - 1), mx[k] + lx - (MSP - 1)
                col, mir = half_col(m, ny), False
                row = wrap_row(mxm, nx) if col >= 0 else -1
                if col < 0:
                    col, row, mir = half_col(-m, ny), wrap_row(-mxm, nx), True
                if col >= 0 and row >= 0:
                    g = grid[row, col]
                    ref += wx[k, lx] * wy[k, ly] * (g.real + 1j * (g.imag if mir else -g.imag))
        # window of virtual cells of the point's 8 x 8 tile
        x0, y0 = mx[k] - (MSP - 1), my[k] - (MSP - 1)
        r0, c0 = (x0 // 8) * 8, (y0 // 8) * 8
        win = np.zeros((32, 32), complex)
        for a in range(32):
            for b in range(32):
                vr, vc = r0 + a, c0 + b
                col = half_col(vc, ny)
                if col >= 0:
                    row = wrap_row(vr, nx)
                    if row >= 0:
                        win[a, b] = np.conj(grid[row, col])
                else:
                    col, row = half_col(-vc, ny), wrap_row(-vr, nx)
                    if col >= 0 and row >= 0:
                        win[a, b] = grid[row, col]
        fx = np.zeros(32)
        fy = np.zeros(32)
        fx[x0 - r0:x0 - r0 + TAPS] = wx[k]
        fy[y0 - c0:y0 - c0 + TAPS] = wy[k]
        val = fx @ win @ fy
        assert abs(val - ref) <= 1e-12 * max(1.0, abs(ref))


def test_spreading_virtual_points_equal_per_cell_rule():
    nx = ny = 16
    mx, my, wx, wy, rng = _case(nx, 40, 3)
    r = rng.standard_normal(len(mx)) + 1j * rng.standard_normal(len(mx))
    G1 = np.zeros((2 * nx, ny + 1), complex)
    for row in range(2 * nx):
        for col in range(ny + 1):
            mrow = row if row < nx else row - 2 * nx
            mcol = col if col < ny else -ny
            for k in range(len(mx)):
                ox, oy = MSP - 1 - mx[k], MSP - 1 - my[k]
                lxd, lyd, lxm, lym = mrow + ox, mcol + oy, ox - mrow, oy - mcol
                if 0 <= lxd < TAPS and 0 <= lyd < TAPS:
                    G1[row, col] += 0.5 * wy[k, lyd] * wx[k, lxd] * np.conj(r[k])
                if 0 <= lxm < TAPS and 0 <= lym < TAPS:
                    G1[row, col] += 0.5 * wy[k, lym] * wx[k, lxm] * r[k]
    TR, TC = 8, 16
    ntc = -(-(ny + 1) // TC)
    lists = {}
    for k in range(len(mx)):
        for fl in (0, 1):
            x0 = -mx[k] - MSP if fl else mx[k] - (MSP - 1)
            y0 = -my[k] - MSP if fl else my[k] - (MSP - 1)
            trs = {wrap_row(v, nx) // TR for v in range(x0, x0 + TAPS) if wrap_row(v, nx) >= 0}
            tcs = {half_col(v, ny) // TC for v in range(y0, y0 + TAPS) if half_col(v, ny) >= 0}
            for a in trs:
                for b in tcs:
                    lists.setdefault(a * ntc + b, []).append((k, fl, x0, y0))
    G2 = np.zeros_like(G1)
    for t, L in lists.items():
        tr, tc = divmod(t, ntc)
        for row in range(tr * TR, min(tr * TR + TR, 2 * nx)):
            mrow = row if row < nx else row - 2 * nx
            for col in range(tc * TC, min(tc * TC + TC, ny + 1)):
                mcol = col if col < ny else -ny
                for (k, fl, x0, y0) in L:
                    jx, jy = mrow - x0, mcol - y0
                    if 0 <= jx < TAPS and 0 <= jy < TAPS:
                        w = (wx[k, TAPS - 1 - jx] * wy[k, TAPS - 1 - jy]) if fl else (wx[k, jx] * wy[k, jy])
                        G2[row, col] += w * 0.5 * (r[k] if fl else np.conj(r[k]))
    assert np.abs(G1 - G2).max() <= 1e-12 * np.abs(G1).max()
