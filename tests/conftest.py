import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
REFERENCE_C = "/root/reference/c"   # present only where the fixtures are made

# field order of the result arrays stored by tests/golden/make_golden.py
RES_KEYS = ["M", "N", "NX", "NY", "N_active", "maxiter", "ITER", "nonneg", "lambda_l1",
            "lambda_tv", "lambda_tsv", "sq_error", "mean_sq_error", "l1cost", "tvcost",
            "tsvcost", "finalcost", "Lip_const"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: takes tens of seconds on the CPU")


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name))


def res_dict(arr):
    return {k: float(v) for k, v in zip(RES_KEYS, arr)}


def rel(a, b):
    """Relative L2 error of a against b (complex inputs compared as complex)."""
    cplx = np.iscomplexobj(a) or np.iscomplexobj(b)
    a = np.asarray(a, np.complex128 if cplx else np.float64)
    b = np.asarray(b, np.complex128 if cplx else np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.fixture(scope="session")
def c0():
    return load_golden("c0_nufft.npz")


@pytest.fixture(scope="session")
def c1():
    return load_golden("c1_fft.npz")


@pytest.fixture(scope="session")
def c2():
    return load_golden("c2_dft_small.npz")


@pytest.fixture(scope="session")
def gpulib():
    """The CUDA library, built in-tree if stale (GPU tests only)."""
    from sparseimaging_b200 import build
    build.build(verbose=False)
    import sparseimaging_b200 as si
    si.lib()
    os.environ.setdefault("MFISTA_QUIET", "1")
    return si
