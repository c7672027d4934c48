"""The leave-one-out error oracle (oracle/looe_oracle.py) against the
reference's own code (c/looe_lib.c compiled into oracle/_ref), through the
committed fixture tests/golden/looe_small.npz and, where oracle/_ref is
built, directly on further seeded problems."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..")
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
from oracle import looe_oracle as O  # noqa: E402
import make_looe_golden as G  # noqa: E402


def _golden():
    d = np.load(os.path.join(ROOT, "tests", "golden", "looe_small.npz"))
    y, A, x, nx = d["y"], d["A"], d["x"], int(d["nx"])
    return y, A, x, nx, {k[:-4]: d[k] for k in d.files if k.endswith("_out")}


def test_restatement_matches_reference_fixture():
    y, A, x, nx, want = _golden()
    for name, (Ac, xc, lt) in G.cases(y, A, x).items():
        st, m, sd = O.looe(y, Ac, xc, nx, lt)
        assert st == want[name][0], name
        if st:
            assert abs(m - want[name][1]) <= 1e-12 * want[name][1], name
            assert abs(sd - want[name][2]) <= 1e-12 * want[name][2], name
        else:
            assert m == 0.0 and sd == 0.0


@pytest.mark.skipif(not os.path.exists(O.REF_LIB), reason="oracle/_ref not built")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_restatement_matches_reference_code(seed):
    rng = np.random.default_rng(seed)
    nx = 10
    M, N = 150, nx * nx
    A = rng.normal(size=(M, N))
    x = np.where(rng.random(N) < 0.4, rng.normal(size=N), 0.0)
    y = A @ x + 0.05 * rng.normal(size=M)
    for lt in (0.0, 0.3):
        a = O.looe(y, A, x, nx, lt)
        b = O.looe_ref(y, A, x, nx, nx, 1.0, lt)
        assert a[0] == b[0] == 1
        assert abs(a[1] - b[1]) <= 1e-11 * b[1] and abs(a[2] - b[2]) <= 1e-11 * b[2]
