"""Regenerate tests/golden/adjoint_clustered.npz:

    python tests/golden/make_adjoint_golden.py

Gradients dL/dD, dL/dE of L = sum_i g_i lambda_i (eigenvalues ascending)
for the seeded "clustered" family at n = 32 and 96, from eigenvectors
computed with mpmath at 50 significant digits:
    dL/dD_i = sum_j g_j v_ij^2,  dL/dE_i = 2 sum_j g_j v_ij v_i+1,j.
These spectra have gaps down to ~1e-13, where double-precision eigenvectors
(LAPACK's included) carry errors of order eps/gap, so a double-precision
reference cannot pin the adjoint there.  g is numpy default_rng(7) normals.
"""
import os
import sys

import mpmath
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "ppopp27-brdc-ae_b200"))
from brdc import families  # noqa: E402

ORDERS = (32, 96)


def exact_grads(d, e, g):
    n = len(d)
    mpmath.mp.dps = 50
    A = mpmath.matrix(n, n)
    for i in range(n):
        A[i, i] = mpmath.mpf(d[i])
        if i + 1 < n:
            A[i, i + 1] = A[i + 1, i] = mpmath.mpf(e[i])
    w, Q = mpmath.eigsy(A)
    order = sorted(range(n), key=lambda j: w[j])
    gd = [mpmath.mpf(0)] * n
    ge = [mpmath.mpf(0)] * (n - 1)
    for r, j in enumerate(order):
        gr = mpmath.mpf(g[r])
        for i in range(n):
            gd[i] += gr * Q[i, j] ** 2
        for i in range(n - 1):
            ge[i] += 2 * gr * Q[i, j] * Q[i + 1, j]
    return np.array([float(x) for x in gd]), np.array([float(x) for x in ge])


def main() -> None:
    out = {}
    for n in ORDERS:
        d, e = families.generate("clustered", n)
        g = np.random.default_rng(7).standard_normal(n)
        gd, ge = exact_grads(d, e, g)
        out[f"gd{n}"] = gd
        out[f"ge{n}"] = ge
        out[f"g{n}"] = g
    np.savez(os.path.join(HERE, "adjoint_clustered.npz"), **out)


if __name__ == "__main__":
    main()
