"""Writes tests/golden/looe_small.npz: the reference's own leave-one-out
error (c/looe_lib.c compute_LOOE_L1 / compute_LOOE_L1_TSV, compiled into
oracle/_ref/liblooe_ref.so by oracle/Makefile) on seeded small problems.

    make -C oracle && python tests/golden/make_looe_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
from oracle import looe_oracle as O  # noqa: E402


def problem():
    rng = np.random.default_rng(11)
    nx, M = 8, 90
    N = nx * nx
    A = rng.normal(size=(M, N))
    x = np.where(rng.random(N) < 0.3, rng.random(N), 0.0)
    y = A @ x + 0.1 * rng.normal(size=M)
    return y, A, x, nx


def cases(y, A, x):
    """name -> (A, x, lambda_tsv): L1 and TSV forms, a Hessian that is not
    positive definite (an active column of A set to zero: a zero pivot in
    any order of operations), an empty active set."""
    A0 = A.copy()
    A0[:, np.flatnonzero(x)[1]] = 0.0
    return {"l1": (A, x, 0.0), "tsv": (A, x, 0.7), "singular": (A0, x, 0.0), "empty": (A, np.zeros_like(x), 0.0)}


def main():
    y, A, x, nx = problem()
    out = {"y": y, "A": A, "x": x, "nx": nx}
    for name, (Ac, xc, lt) in cases(y, A, x).items():
        st, m, sd = O.looe_ref(y, Ac, xc, nx, nx, 1.0, lt)
        out[f"{name}_out"] = np.array([st, m, sd])
    np.savez_compressed(os.path.join(HERE, "looe_small.npz"), **out)


if __name__ == "__main__":
    main()
