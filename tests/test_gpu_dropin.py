"""The reference's own command-line drivers, linked against this library.

oracle/_ref/dropin_{nufft,fft,dft} are c/mfista_imaging_{nufft,fft,dft}.c
with their I/O and allocation helpers (c/mfista_io.c, c/mfista_tools.c),
compiled unchanged and linked against sparseimaging_b200/libmfista_b200.so
in place of the reference solver objects (`make -C oracle dropin`, run by
__graft_entry__.build()).  Each test writes an input file in the driver's
own format, runs the driver as a user would, and compares the image it
writes (raw doubles, c/mfista_io.c write_X_vector) and the summary it
prints (c/mfista_io.c show_result) with the reference's output on the same
input: the reference's sample data (c/nufft_data.txt, c/fft_data.txt;
tests/golden/make_refdata_golden.py) and the small DFT fixture.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, rel, res_dict

pytestmark = pytest.mark.gpu

REF_OUT = os.path.join(ROOT, "oracle", "_ref")


def _driver(name):
    path = os.path.join(REF_OUT, f"dropin_{name}")
    if not os.path.exists(path):
        pytest.fail(f"{path} is not built (make -C oracle dropin)")
    return path


def _run(args, cwd):
    env = dict(os.environ)
    env.pop("MFISTA_QUIET", None)
    p = subprocess.run(args, cwd=cwd, capture_output=True, text=True, timeout=600, env=env)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    return p.stdout


def _summary(out):
    it = int(re.search(r"# of iterations:\s+(\d+)", out).group(1))
    cost = float(re.search(r"cost:\s+([-+0-9.eE]+)", out).group(1))
    return it, cost


def _write_nufft(path, g):
    with open(path, "w") as f:
        f.write(f"M  = {g['u'].size}\nNX = {int(g['nx'])}\nNY = {int(g['ny'])}\n\n")
        f.write("u_rad, v_rad, vis_r, vis_i, noise_std_dev\n\n")
        for row in zip(g["u"], g["v"], g["vis_r"], g["vis_i"], g["vis_std"]):
            f.write(", ".join(f"{v:.17e}" for v in row) + "\n")


def _write_fft(path, g):
    with open(path, "w") as f:
        f.write(f"M  = {g['u_idx'].size}\nNX = {int(g['nx'])}\nNY = {int(g['ny'])}\n\n")
        f.write("u, v, y_r, y_i, noise_std_dev\n\n")
        for a, b, c, d, e in zip(g["u_idx"], g["v_idx"], g["y_r"], g["y_i"], g["noise"]):
            f.write(f"{int(a)}, {int(b)}, {c:.17e}, {d:.17e}, {e:.17e}\n")


def test_dropin_nufft_driver(tmp_path):
    """mfista_imaging_nufft on the reference's nufft_data.txt with the
    parameters of matlab/testdata4nufft.mat, 30 iterations (the solve is
    chaotic under 1-ulp changes from about iteration 60 on)."""
    g = np.load(os.path.join(GOLDEN, "refdata_nufft.npz"))
    data = tmp_path / "nufft_data.txt"
    _write_nufft(data, g)
    out = _run([_driver("nufft"), str(data), "100", "0", "100", "5e8", "x.out", "-nonneg", "-maxiter", "30",
                "-eps", "1e-3"], tmp_path)
    x = np.fromfile(tmp_path / "x.out", dtype=np.float64)
    gold = res_dict(g["short_res"])
    it, cost = _summary(out)
    assert x.size == int(g["nx"]) * int(g["ny"])
    assert it == gold["ITER"] == 30
    assert rel(x, g["short_x"]) < 1e-7
    assert abs(cost - gold["finalcost"]) <= 1e-6 * gold["finalcost"]  # printed with %e


def test_dropin_fft_driver(tmp_path):
    """mfista_imaging_fft on the reference's fft_data.txt, L1+TSV to the
    default stopping rule."""
    g = np.load(os.path.join(GOLDEN, "refdata_fft.npz"))
    data = tmp_path / "fft_data.txt"
    _write_fft(data, g)
    out = _run([_driver("fft"), str(data), "1", "0", "0.01", "5e10", "x.out", "-nonneg"], tmp_path)
    x = np.fromfile(tmp_path / "x.out", dtype=np.float64)
    gold = res_dict(g["tsv_res"])
    it, cost = _summary(out)
    assert it == gold["ITER"]
    assert rel(x, g["tsv_x"]) < 1e-7
    assert abs(cost - gold["finalcost"]) <= 1e-6 * gold["finalcost"]


def test_dropin_dft_driver(tmp_path, c2):
    """mfista_imaging_dft with the DFT fixture's y and column-major A as raw
    double files, L1+TSV, 300 iterations."""
    A = np.asarray(c2["A"])
    m, n = A.shape
    np.asarray(c2["y"], np.float64).tofile(tmp_path / "y.bin")
    np.asfortranarray(A).ravel(order="F").tofile(tmp_path / "A.bin")
    lam1 = float(c2["lam1"])
    out = _run([_driver("dft"), str(m), str(n), "y.bin", "A.bin", repr(lam1), "0", repr(1e-3 * lam1),
                repr(float(c2["cinit"])), "x.out", "-nonneg", "-maxiter", "300", "-eps", "1e-6"], tmp_path)
    x = np.fromfile(tmp_path / "x.out", dtype=np.float64)
    gold = res_dict(c2["tsv_res"])
    it, cost = _summary(out)
    assert it == gold["ITER"]
    assert rel(x, c2["tsv_x"]) < 1e-7
    assert abs(cost - gold["finalcost"]) <= 1e-6 * gold["finalcost"]
