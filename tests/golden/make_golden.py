"""Generate the golden fixtures of the reference's known-answer test.

fastSolver's only results-pinning check (test/single_launch.cc:20-75,
src/solver/direct_solve.cc:129-231) solves A = diag*I + U U^T, with circulant
U(i, j) = (i + j) mod r and a drand48_r right-hand side reseeded for every
leaf region, both densely and with the HODLR solver, and prints the relative
Frobenius difference.  This script restates that dense side independently of
the oracle (numpy only: glibc's drand48 recurrence, the circulant formula,
numpy.linalg.solve) and stores the right-hand side and the dense solution:

  kat_n480.npz   the reference run itself: N=480, r=30, threshold=60, m=2,
                 diag=1e4, seed=1245667 (8 leaves of 60 rows)
  kat_n201.npz   an unbalanced tree: N=201, threshold=100 -> leaves of 100,
                 50 and 51 rows at depths 1 and 2; r=10, m=3, diag=1e3
  kat_n1000.npz  N=1000, r=20, threshold=128, m=4, diag=5e2 (leaves of 125)

Run: python tests/golden/make_golden.py
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

CASES = {
    "kat_n480": dict(N=480, nrhs=2, rank=30, threshold=60, diag=1.0e4, seed=1245667),
    "kat_n201": dict(N=201, nrhs=3, rank=10, threshold=100, diag=1.0e3, seed=7),
    "kat_n1000": dict(N=1000, nrhs=4, rank=20, threshold=128, diag=5.0e2, seed=99),
}


def leaf_ranges(N: int, threshold: int):
    """(row_beg, nrow) of the leaves, left to right: split N/2, N - N/2."""
    out = []

    def rec(rb, n):
        if n > threshold:
            rec(rb, n // 2)
            rec(rb + n // 2, n - n // 2)
        else:
            out.append((rb, n))

    rec(0, N)
    return out


def drand48_block(seed: int, nrow: int, ncol: int) -> np.ndarray:
    x = ((seed & 0xFFFFFFFF) << 16) | 0x330E
    a, c, mask = 0x5DEECE66D, 0xB, (1 << 48) - 1
    out = np.empty((nrow, ncol))
    for i in range(nrow):
        for j in range(ncol):
            x = (a * x + c) & mask
            out[i, j] = x / float(1 << 48)
    return out


def make(N, nrhs, rank, threshold, diag, seed):
    B = np.zeros((N, nrhs))
    for rb, n in leaf_ranges(N, threshold):
        B[rb:rb + n] = drand48_block(seed, n, nrhs)
    i = np.arange(N)[:, None]
    j = np.arange(rank)[None, :]
    U = ((i + j) % rank).astype(np.float64)
    A = diag * np.eye(N) + U @ U.T
    X = np.linalg.solve(A, B)
    return B, X


def main():
    for name, cfg in CASES.items():
        B, X = make(**cfg)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), B=B, X=X,
                            **{k: np.array(v) for k, v in cfg.items()})
        print(name, B.shape, float(np.abs(X).max()))


if __name__ == "__main__":
    main()
