"""The 50-digit adjoint fixture agrees with double-precision LAPACK
eigenvectors to within LAPACK's own accuracy on these spectra, and its
g vectors are the ones the GPU tests regenerate."""
import os

import numpy as np
import pytest
import scipy.linalg

from brdc import families

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("n", [32, 96])
def test_fixture_matches_lapack_loosely(n):
    ref = np.load(os.path.join(GOLDEN, "adjoint_clustered.npz"))
    d, e = families.generate("clustered", n)
    g = ref[f"g{n}"]
    assert np.array_equal(g, np.random.default_rng(7).standard_normal(n))
    w, V = scipy.linalg.eigh_tridiagonal(d, e)
    rd = (V * V) @ g
    re = 2.0 * (V[:-1] * V[1:]) @ g
    sc = max(np.max(np.abs(rd)), np.max(np.abs(re)))
    assert np.max(np.abs(ref[f"gd{n}"] - rd)) < 1e-5 * sc
    assert np.max(np.abs(ref[f"ge{n}"] - re)) < 1e-8 * sc
    # trace identity: sum_i dL/dD_i = sum_j g_j (each v_j has unit norm)
    assert abs(ref[f"gd{n}"].sum() - g.sum()) < 1e-12 * np.abs(g).sum()
