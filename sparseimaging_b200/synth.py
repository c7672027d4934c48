"""Seeded synthetic skies, uv coverages and visibilities.

The reference ships no benchmark suite and publishes no dataset for its
solver path; these generators stand in for one.  They produce inputs in the
reference's own argument conventions:

* NUFFT variant (c/mfista_nufft_lib.c:909): ``u_dx, v_dy`` in radians per
  pixel, ``vis_r, vis_i, vis_std`` per uv point, image ``x[i*Ny + j]``.
  The forward model is the one the reference's gridding approximates
  (c/mfista_nufft_lib.c:187-243 with the centred padding of :42-48 and
  NU_SIGN = -1 at :27):
      V(u, v) = sum_ij x[i, j] * exp(+1j * (u * (i - Nx/2) + v * (j - Ny/2))).
* FFT variant (c/mfista_fft_lib.c:701): integer cells ``u_idx, v_idx`` in
  [0, NX) x [0, NY) with every Hermitian partner present (the cost divides a
  full-plane norm by 4, c/mfista_fft_lib.c:158).
* DFT variant (c/mfista_dft_lib.c:540): a real column-major M x N matrix
  obtained by stacking real and imaginary rows, weights applied.

Everything is seeded with ``numpy.random.default_rng(seed)``.
"""
from __future__ import annotations

import dataclasses
import numpy as np


# --------------------------------------------------------------------------
# skies
# --------------------------------------------------------------------------

def _gauss(n, cx, cy, sigma):
    i = np.arange(n)[:, None]
    j = np.arange(n)[None, :]
    return np.exp(-((i - cx) ** 2 + (j - cy) ** 2) / (2.0 * sigma ** 2))


def sky_blobs_ring(n, seed, n_blobs=3, sigma=(2.0, 6.0), peak=(0.2, 1.0),
                   ring_radius=12.0, ring_width=2.0, ring_amp=0.5,
                   ring_axes=None, rng=None):
    """Gaussian blobs plus a ring; clipped >= 0; total flux 1.

    ``ring_axes=(a, b)`` gives an elliptical ring with those semi-axes.
    Returns an (n, n) float64 array indexed [i, j] (reference layout i*Ny+j).
    """
    rng = np.random.default_rng(seed) if rng is None else rng
    img = np.zeros((n, n))
    lo, hi = 0.125 * n, 0.875 * n
    for _ in range(n_blobs):
        cx, cy = rng.uniform(lo, hi, size=2)
        s = rng.uniform(*sigma)
        a = rng.uniform(*peak)
        img += a * _gauss(n, cx, cy, s)
    if ring_amp > 0:
        c = n / 2.0
        i = np.arange(n)[:, None] - c
        j = np.arange(n)[None, :] - c
        if ring_axes is None:
            r = np.sqrt(i ** 2 + j ** 2)
            img += ring_amp * np.exp(-((r - ring_radius) ** 2) / (2.0 * ring_width ** 2))
        else:
            a, b = ring_axes
            rr = np.sqrt((i / a) ** 2 + (j / b) ** 2)
            img += ring_amp * np.exp(-(((rr - 1.0) * 0.5 * (a + b)) ** 2) / (2.0 * ring_width ** 2))
    img = np.clip(img, 0.0, None)
    return img / img.sum()


def sky_movie_frame(n, frame, seed=3, ring_radius=24.0, spot_step_deg=7.5):
    """Ring with a bright spot rotating ``spot_step_deg`` per frame + 2 static blobs."""
    rng = np.random.default_rng(seed)
    c = n / 2.0
    i = np.arange(n)[:, None] - c
    j = np.arange(n)[None, :] - c
    r = np.sqrt(i ** 2 + j ** 2)
    img = 0.5 * np.exp(-((r - ring_radius) ** 2) / (2.0 * 2.0 ** 2))
    ang = np.deg2rad(spot_step_deg * frame)
    img += 1.0 * _gauss(n, c + ring_radius * np.cos(ang), c + ring_radius * np.sin(ang), 3.0)
    for _ in range(2):
        cx, cy = rng.uniform(0.2 * n, 0.8 * n, size=2)
        img += rng.uniform(0.2, 0.6) * _gauss(n, cx, cy, rng.uniform(2.0, 5.0))
    img = np.clip(img, 0.0, None)
    return img / img.sum()


def sky_training(n, seed):
    """3-12 blobs (sigma 1-10 px) plus, w.p. 0.5, a ring or a crescent; flux 1."""
    rng = np.random.default_rng(seed)
    img = np.zeros((n, n))
    for _ in range(int(rng.integers(3, 13))):
        cx, cy = rng.uniform(0.15 * n, 0.85 * n, size=2)
        img += rng.uniform(0.1, 1.0) * _gauss(n, cx, cy, rng.uniform(1.0, 10.0))
    if rng.random() < 0.5:
        c = n / 2.0 + rng.uniform(-0.1, 0.1, size=2) * n
        rad = rng.uniform(0.08, 0.2) * n
        i = np.arange(n)[:, None] - c[0]
        j = np.arange(n)[None, :] - c[1]
        r = np.sqrt(i ** 2 + j ** 2)
        ring = np.exp(-((r - rad) ** 2) / (2.0 * (0.02 * n) ** 2))
        if rng.random() < 0.5:  # crescent: brightness modulated by angle
            th = np.arctan2(j, i) - rng.uniform(0, 2 * np.pi)
            ring *= 0.5 * (1.0 + np.cos(th))
        img += rng.uniform(0.3, 1.0) * ring
    img = np.clip(img, 0.0, None)
    return img / img.sum()


# --------------------------------------------------------------------------
# uv coverage
# --------------------------------------------------------------------------

def safe_kmax(nx):
    """Largest |k| (cycles per field of view) the reference gridding keeps in
    bounds: mx = round(2k) and mx + 12 must stay below Nx
    (c/mfista_nufft_lib.c:32-40 maps m >= Mr/2 out of the array)."""
    return (nx - 14) // 2


def earth_rotation_uv(n_stations, n_hours, seed, dec_deg=45.0, span_hours=12.0, rng=None):
    """Stations uniform in the unit disk; every baseline traces an
    Earth-rotation ellipse u = bx sin h + by cos h, v = sin(dec)(-bx cos h + by sin h)."""
    rng = np.random.default_rng(seed) if rng is None else rng
    r = np.sqrt(rng.uniform(0, 1, n_stations))
    th = rng.uniform(0, 2 * np.pi, n_stations)
    pos = np.stack([r * np.cos(th), r * np.sin(th)], axis=1)
    h = np.linspace(-0.5, 0.5, n_hours) * (span_hours / 24.0) * 2 * np.pi
    sd = np.sin(np.deg2rad(dec_deg))
    us, vs = [], []
    for a in range(n_stations):
        for b in range(a + 1, n_stations):
            bx, by = pos[b] - pos[a]
            us.append(bx * np.sin(h) + by * np.cos(h))
            vs.append(sd * (-bx * np.cos(h) + by * np.sin(h)))
    return np.concatenate(us), np.concatenate(vs)


def scale_uv_to_radians(u, v, nx, kmax):
    """Scale so max(|u|,|v|) = kmax cycles per FOV; return radians per pixel."""
    s = kmax / max(np.abs(u).max(), np.abs(v).max())
    return 2 * np.pi * u * s / nx, 2 * np.pi * v * s / nx


def dft_vis(x, u_dx, v_dy):
    """Exact visibilities of image x (nx, ny) at (u_dx, v_dy) radians/pixel."""
    nx, ny = x.shape
    ex = np.exp(1j * np.outer(u_dx, np.arange(nx) - nx // 2))
    ey = np.exp(1j * np.outer(v_dy, np.arange(ny) - ny // 2))
    return np.einsum("ki,ij,kj->k", ex, x.astype(np.complex128), ey, optimize=True)


# --------------------------------------------------------------------------
# problem bundles
# --------------------------------------------------------------------------

@dataclasses.dataclass
class NufftProblem:
    u_dx: np.ndarray
    v_dy: np.ndarray
    vis_r: np.ndarray
    vis_i: np.ndarray
    vis_std: np.ndarray
    nx: int
    ny: int
    sky: np.ndarray

    @property
    def m(self):
        return int(self.u_dx.size)


def nufft_problem(nx, n_stations, n_hours, seed, noise_frac=0.01, kmax=None,
                  sky=None, dec_deg=45.0, span_hours=12.0):
    rng = np.random.default_rng(seed)
    if sky is None:
        sky = sky_blobs_ring(nx, seed=None, rng=rng,
                             ring_radius=12.0 * nx / 64.0, ring_width=2.0 * nx / 64.0)
    u, v = earth_rotation_uv(n_stations, n_hours, seed=None, rng=rng,
                             dec_deg=dec_deg, span_hours=span_hours)
    u_dx, v_dy = scale_uv_to_radians(u, v, nx, safe_kmax(nx) if kmax is None else kmax)
    vis = dft_vis(sky, u_dx, v_dy)
    sigma = noise_frac * np.abs(vis).max()
    vis = vis + sigma * (rng.standard_normal(vis.size) + 1j * rng.standard_normal(vis.size))
    std = np.full(vis.size, sigma)
    return NufftProblem(u_dx, v_dy, vis.real.copy(), vis.imag.copy(), std, nx, nx, sky)


def config0(seed=0):
    """64x64, 8 stations x 72 hour angles (M = 2016), 1 % noise."""
    return nufft_problem(64, 8, 72, seed)


def movie_problem(n_frames=48, nx=128, seed=3, m_range=(800, 12000), noise_frac=0.02):
    """Frames of a movie with uneven visibility counts: frame f shows
    sky_movie_frame(nx, f) (the ring's bright spot turns 7.5 degrees per
    frame, two static blobs); its uv coverage has 6-10 stations and as many
    hour angles over 12 h as bring M = baselines x hours near a value drawn
    uniformly from m_range.  Noise: noise_frac of max|V| per frame."""
    rng = np.random.default_rng(seed)
    frames = []
    for f in range(n_frames):
        ns = int(rng.integers(6, 11))
        nb = ns * (ns - 1) // 2
        m_goal = rng.uniform(*m_range)
        nh = max(1, int(round(m_goal / nb)))
        sky = sky_movie_frame(nx, f, seed=seed)
        frames.append(nufft_problem(nx, ns, nh, int(rng.integers(1 << 30)), noise_frac=noise_frac, sky=sky))
    return frames


def lambda_grid_problem(seed=7, nx=128, n_stations=10, n_hours=180):
    """128x128 NUFFT problem (M = 45 * 180 = 8100) shared by a lambda grid."""
    return nufft_problem(nx, n_stations, n_hours, seed)


def lambda_grid(max_grad, n1=8, n2=8, lo=1e-4, hi=1.0, tsv_ratio=None):
    """n1 x n2 log grid of (lambda_l1, lambda_tsv) spanning lo..hi of max|A^H y|."""
    l1 = np.logspace(np.log10(lo), np.log10(hi), n1) * max_grad
    if tsv_ratio is None:
        lt = np.logspace(np.log10(lo), np.log10(hi), n2) * max_grad
    else:
        lt = None
    pairs = []
    for a in range(n1):
        for b in range(n2):
            pairs.append((l1[a], (lt[b] if lt is not None else tsv_ratio * l1[a])))
    return np.array(pairs)


@dataclasses.dataclass
class FftProblem:
    u_idx: np.ndarray
    v_idx: np.ndarray
    y_r: np.ndarray
    y_i: np.ndarray
    noise_stdev: np.ndarray
    nx: int
    ny: int
    sky: np.ndarray


def fft_problem(nx=128, n_cells=3000, seed=1, r_lo=4.0, r_hi=60.0, noise_frac=0.01,
                n_blobs=6, ring_axes=(20.0, 16.0)):
    """Gridded visibilities on ``n_cells`` distinct half-plane cells from the
    annulus r_lo..r_hi, each written together with its Hermitian partner.

    Values are the model of c/mfista_fft_lib.c:142-159: F = FFT2(x)/sqrt(N)
    (forward sign, unnormalised FFT scaled by 1/sqrt(N))."""
    rng = np.random.default_rng(seed)
    sky = sky_blobs_ring(nx, seed=None, rng=rng, n_blobs=n_blobs, ring_axes=ring_axes,
                         ring_width=2.0)
    ny = nx
    ks = []
    for a in range(-nx // 2 + 1, nx // 2):
        for b in range(0, ny // 2):
            r = np.hypot(a, b)
            if not (r_lo <= r <= r_hi):
                continue
            if b == 0 and a <= 0:  # keep one cell of each conjugate pair
                continue
            ks.append((a, b))
    ks = np.array(ks)
    sel = ks[rng.choice(len(ks), size=n_cells, replace=False)]
    F = np.fft.fft2(sky) / np.sqrt(nx * ny)
    ua = np.concatenate([sel[:, 0] % nx, (-sel[:, 0]) % nx])
    va = np.concatenate([sel[:, 1] % ny, (-sel[:, 1]) % ny])
    vals = F[ua[:n_cells], va[:n_cells]]
    sigma = noise_frac * np.abs(vals).max()
    noise = sigma * (rng.standard_normal(n_cells) + 1j * rng.standard_normal(n_cells))
    vals = vals + noise
    vals = np.concatenate([vals, np.conj(vals)])
    std = np.full(2 * n_cells, sigma)
    return FftProblem(ua.astype(np.int32), va.astype(np.int32), vals.real.copy(),
                      vals.imag.copy(), std, nx, ny, sky)


@dataclasses.dataclass
class DftProblem:
    y: np.ndarray      # [M_real]
    A: np.ndarray      # column-major M_real x N, as a Fortran-ordered array
    nx: int
    ny: int
    sky: np.ndarray


def dft_problem(nx=64, n_stations=10, n_hours=89, seed=2, noise_frac=0.01, m_vis=4000):
    """Real-stacked weighted DFT matrix [Re; Im] * diag(1/sigma) (c/mfista_dft_lib.c:30-66)."""
    rng = np.random.default_rng(seed)
    sky = sky_blobs_ring(nx, seed=None, rng=rng, ring_radius=12.0 * nx / 64.0,
                         ring_width=2.0 * nx / 64.0)
    u, v = earth_rotation_uv(n_stations, n_hours, seed=None, rng=rng)
    u, v = u[:m_vis], v[:m_vis]
    u_dx, v_dy = scale_uv_to_radians(u, v, nx, nx // 2)
    ex = np.exp(1j * np.outer(u_dx, np.arange(nx) - nx // 2))
    ey = np.exp(1j * np.outer(v_dy, np.arange(nx) - nx // 2))
    Ac = (ex[:, :, None] * ey[:, None, :]).reshape(u_dx.size, nx * nx)
    vis = Ac @ sky.reshape(-1)
    sigma = noise_frac * np.abs(vis).max()
    vis = vis + sigma * (rng.standard_normal(vis.size) + 1j * rng.standard_normal(vis.size))
    w = 1.0 / sigma
    A = np.asfortranarray(np.concatenate([Ac.real, Ac.imag], axis=0) * w)
    y = np.concatenate([vis.real, vis.imag]) * w
    return DftProblem(y, A, nx, nx, sky)
