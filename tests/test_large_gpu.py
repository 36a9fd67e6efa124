"""Orders above the headline size, where the upper merges are larger than one
4096-position chunk of k_level's merge path and placement (the chunk loop,
its split searches and the staged ranges of later chunks all run), and an
odd order whose tree is uneven at every level.  Eigenvalues are checked at
sampled indices (both ends included) against LAPACK's bisection (DSTEBZ via
scipy), the whole spectrum against its trace and Frobenius norm, and the
Toeplitz closed form over every eigenvalue."""
import numpy as np
import pytest

from brdc import families

pytestmark = pytest.mark.gpu
TOL = 1e-12  # max |lambda - lambda_ref| / ||T||_2


def gpu_solve(solver, d, e):
    import torch

    W = solver.dstebr(torch.tensor(d, device="cuda"), torch.tensor(e, device="cuda"))
    assert solver.info(len(d)) == 0
    return W.cpu().numpy()


def sampled_reference(d, e, idx):
    from scipy.linalg import eigvalsh_tridiagonal

    return np.array([eigvalsh_tridiagonal(d, e, select="i", select_range=(int(i), int(i)),
                                          lapack_driver="stebz")[0] for i in idx])


@pytest.mark.parametrize("family,n", [("uniform", 262144), ("normal", 200003)])
def test_large_orders_sampled(solver, family, n):
    d, e = families.generate(family, n)
    w = gpu_solve(solver, d, e)
    assert np.all(np.diff(w) >= 0.0)
    idx = np.unique(np.concatenate([[0, 1, n - 2, n - 1],
                                    np.linspace(0, n - 1, 60).astype(np.int64)]))
    ref = sampled_reference(d, e, idx)
    scale = max(np.abs(w[0]), np.abs(w[-1]))
    assert np.max(np.abs(w[idx] - ref)) < TOL * scale
    assert abs(w.sum() - d.sum()) < 1e-10 * np.abs(w).sum()
    assert abs((w * w).sum() - (d * d).sum() - 2 * (e * e).sum()) < 1e-10 * (w * w).sum()


def test_large_toeplitz_closed_form(solver):
    n = 131072
    d, e = families.generate("toeplitz", n)
    w = gpu_solve(solver, d, e)
    ref = families.toeplitz_eigenvalues(n)
    assert np.max(np.abs(w - ref)) < TOL * 4.0
