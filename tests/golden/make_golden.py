"""Generate tests/golden/dgbsv_cases.npz: banded systems solved by LAPACK dgbsv as shipped
in scipy's bundled OpenBLAS (the library GEMINI3D links as LAPACK when built against
OpenBLAS).  The oracle's restated dgbtf2/dgbtrs is checked against these vectors.

Cases: random diagonally dominant and random general kl=ku=2 systems, and the TRBDF2
matrices of PDEparabolic.f90 (identity Dirichlet rows, stiff conduction rows) that force
LAPACK's row interchanges.

    python tests/golden/make_golden.py
"""
import os

import numpy as np
from scipy.linalg import lapack

HERE = os.path.dirname(os.path.abspath(__file__))


def band(A, kl, ku):
    n = A.shape[0]
    ab = np.zeros((2 * kl + ku + 1, n), order="F")
    for j in range(n):
        for i in range(max(0, j - ku), min(n, j + kl + 1)):
            ab[kl + ku + i - j, j] = A[i, j]
    return ab


def trbdf2_matrix(n, s, dt, rng):
    A = np.zeros((n, n))
    A[0, 0] = A[-1, -1] = 1.0
    for i in range(1, n - 1):
        lo, up = -s * rng.uniform(0.5, 2.0), -s * rng.uniform(0.5, 2.0)
        A[i, i - 1], A[i, i + 1], A[i, i] = lo, up, 2 / dt - lo - up
    return A


def main():
    rng = np.random.default_rng(2024)
    abs_, bs, xs, pivs, ns = [], [], [], [], []
    systems = []
    for n in (8, 17, 64):
        A = np.zeros((n, n))
        for i in range(n):
            for j in range(max(0, i - 2), min(n, i + 3)):
                A[i, j] = rng.standard_normal()
        systems.append(A)
        D = A.copy()
        D[np.arange(n), np.arange(n)] = np.abs(A).sum(1) + 1
        systems.append(D)
    for s in (10.0, 3e4, 1e8):
        systems.append(trbdf2_matrix(40, s, 0.7, rng))
    n_max = max(A.shape[0] for A in systems)
    for A in systems:
        n = A.shape[0]
        ab = band(A, 2, 2)
        b = rng.standard_normal(n) * 100
        lu, piv, x, info = lapack.dgbsv(2, 2, ab.copy(order="F"), b.copy())
        assert info == 0
        pad = lambda v, m: np.concatenate([v, np.zeros(m - len(v))])
        abs_.append(np.pad(ab, ((0, 0), (0, n_max - n))))
        bs.append(pad(b, n_max))
        xs.append(pad(x, n_max))
        pivs.append(np.pad(piv, (0, n_max - n)))
        ns.append(n)
    np.savez(os.path.join(HERE, "dgbsv_cases.npz"), ab=np.array(abs_), b=np.array(bs), x=np.array(xs),
             piv=np.array(pivs), n=np.array(ns))


if __name__ == "__main__":
    main()
