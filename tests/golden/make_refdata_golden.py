"""Golden fixtures of full solves on the reference's own sample data.

Run here (where the reference sources exist) after `make -C oracle`:

    python tests/golden/make_refdata_golden.py

The reference ships two data files for its command-line drivers,
c/nufft_data.txt (M = 7648 uv points, 200 x 200 image) and c/fft_data.txt
(M = 6590 gridded cells, 128 x 128 image), and one parameter set for the
NUFFT data (matlab/testdata4nufft.mat: lambda_l1 = 100, lambda_tsv = 100,
cinit = 5e8, eps = 1e-3, maxiter = 5000, nonnegative).  The FFT data is
solved with the parameters of matlab/test_algorithm.m (lambda_l1 = 1,
lambda_2 = 0.01, cinit = 5e10) as an L1+TSV and as an L1+TV problem, with
the drivers' default eps (1e-5, c/mfista.h:41) and maxiter (50000).

Every solve is the reference C compiled unchanged (oracle/_ref, FFTW/BLAS
shims) through its entry point -- the call the drivers make.  The parsed
data, the parameters, xout and the RESULT fields go into
tests/golden/refdata_{nufft,fft}.npz.  For each solve the reference's own
spread under 1-ulp changes of one visibility is stored too
(`*_envelope_x`, `*_envelope_cost`), the floor any other FFT or summation
order can be held to.  The NUFFT data is solved twice: to the stopping rule
(eps 1e-3; 2365 iterations, chaotic: envelope 3.7e-3 on xout) and for 30
iterations (one trajectory: envelope ~1e-13).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from make_golden import quiet_call, res_arr  # noqa: E402
from oracle import ref_ctypes as R          # noqa: E402

REF_C = "/root/reference/c"


def parse(fname, ints):
    lines = open(fname).read().splitlines()
    m = int(lines[0].split("=")[1])
    nx = int(lines[1].split("=")[1])
    ny = int(lines[2].split("=")[1])
    rows = [[t.strip() for t in ln.split(",")] for ln in lines[6:6 + m]]
    cols = list(zip(*rows))
    out = []
    for k, c in enumerate(cols):
        out.append(np.array([int(v) for v in c], np.int32) if (ints and k < 2) else np.array([float(v) for v in c]))
    return m, nx, ny, out


def envelope(call, base_x, base_cost, vis, k_vis):
    """Largest relative change of xout / finalcost of the reference when
    visibility k_vis is scaled by 1 +- 1e-15."""
    dx = dc = 0.0
    for s in (1 + 1e-15, 1 - 1e-15):
        v = vis.copy()
        v[k_vis] *= s
        x2, r2 = call(v)
        dx = max(dx, float(np.linalg.norm(x2 - base_x) / np.linalg.norm(base_x)))
        dc = max(dc, abs(r2.finalcost - base_cost) / base_cost)
    return dx, dc


def make_nufft():
    m, nx, ny, (u, v, vr, vi, vs) = parse(os.path.join(REF_C, "nufft_data.txt"), ints=False)
    prm = dict(lam1=100.0, lamtsv=100.0, cinit=5e8, eps=1e-3, maxiter=5000)
    out = dict(u=u, v=v, vis_r=vr, vis_i=vi, vis_std=vs, nx=nx, ny=ny, **prm)

    def call(vr_, maxiter=prm["maxiter"]):
        return quiet_call(R.core_nufft, u, v, vr_, vi, vs, nx, ny, maxiter, prm["eps"], prm["lam1"], 0.0,
                          prm["lamtsv"], prm["cinit"], nonneg_flag=1)
    # the full run is chaotic under 1-ulp changes from about iteration 60 on
    # (envelope 1e-7 at 60 iterations, 1e-3 at 100); the short run stays on
    # one trajectory (envelope ~1e-13)
    for tag, mi in (("short", 30), ("full", prm["maxiter"])):
        x, res = call(vr, mi)
        out[f"{tag}_x"], out[f"{tag}_res"] = x, res_arr(res)
        ex, ec = envelope(lambda w: call(w, mi), x, res.finalcost, vr, 0)
        out[f"{tag}_envelope_x"], out[f"{tag}_envelope_cost"] = ex, ec
        print(f"nufft {tag}: ITER {res.ITER} cost {res.finalcost:.10e} envelope x {ex:.2e} cost {ec:.2e}", flush=True)
    np.savez_compressed(os.path.join(HERE, "refdata_nufft.npz"), **out)


def make_fft():
    m, nx, ny, (ui, vi_, yr, yi, ns) = parse(os.path.join(REF_C, "fft_data.txt"), ints=True)
    prm = dict(lam1=1.0, lam2=0.01, cinit=5e10, eps=1e-5, maxiter=50000)
    out = dict(u_idx=ui, v_idx=vi_, y_r=yr, y_i=yi, noise=ns, nx=nx, ny=ny, **prm)
    for tag, ltv, lts in (("tsv", 0.0, prm["lam2"]), ("tv", prm["lam2"], 0.0)):
        def call(yr_):
            return quiet_call(R.core_fft, ui, vi_, yr_, yi, ns, nx, ny, prm["maxiter"], prm["eps"], prm["lam1"], ltv,
                              lts, prm["cinit"], nonneg_flag=1)
        x, res = call(yr)
        out[f"{tag}_x"], out[f"{tag}_res"] = x, res_arr(res)
        ex, ec = envelope(call, x, res.finalcost, yr, 0)
        out[f"{tag}_envelope_x"], out[f"{tag}_envelope_cost"] = ex, ec
        print(f"fft {tag}: ITER {res.ITER} cost {res.finalcost:.10e} envelope x {ex:.2e} cost {ec:.2e}", flush=True)
    np.savez_compressed(os.path.join(HERE, "refdata_fft.npz"), **out)


if __name__ == "__main__":
    which = sys.argv[1:] or ["nufft", "fft"]
    if "fft" in which:
        make_fft()
    if "nufft" in which:
        make_nufft()
