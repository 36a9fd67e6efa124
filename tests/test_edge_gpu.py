"""Hard inputs for the solve: extreme scaling, graded diagonals, glued
Wilkinson matrices (clusters of near-degenerate pairs) and a nearly scalar
matrix (almost everything deflates)."""
import numpy as np
import pytest

import oracle
from brdc import families

pytestmark = pytest.mark.gpu


def solve(solver, d, e):
    import torch

    return solver.dstebr(torch.tensor(d, device="cuda"), torch.tensor(e, device="cuda")).cpu().numpy()


def rel_err(w, ref):
    return float(np.max(np.abs(w - ref)) / np.max(np.abs(ref)))


@pytest.mark.parametrize("scale", [1e-300, 1e-150, 1e150, 1e300])
def test_extreme_scaling(solver, scale):
    """Eigenvalues scale exactly with the matrix; the solve must not
    overflow or underflow on the way (z^2/delta^2 and friends)."""
    n = 5000
    d, e = families.generate("uniform", n)
    base = solve(solver, d, e)
    w = solve(solver, d * scale, e * scale)
    assert np.all(np.isfinite(w))
    assert rel_err(w / scale, base) < 1e-13


@pytest.mark.parametrize("n", [100, 3000])
def test_graded_diagonal(solver, n):
    rng = np.random.default_rng(n)
    d = np.logspace(0, -12, n) * rng.choice([-1.0, 1.0], n)
    e = np.logspace(0, -12, n - 1) * 0.5 * rng.uniform(0.5, 1.0, n - 1)
    w = solve(solver, d, e)
    ref = oracle.dstedc_dc_br(d, e)
    assert rel_err(w, ref) < 1e-12


def test_glued_wilkinson(solver):
    """Copies of W21+ glued by 1e-10 couplings: pairs of eigenvalues agree
    to many digits, inside one child and across children."""
    m = 21
    wd = np.abs(np.arange(m) - (m - 1) / 2.0)
    blocks = 150
    d = np.tile(wd, blocks)
    e = np.ones(m * blocks - 1)
    e[m - 1::m] = 1e-10
    w = solve(solver, d, e)
    ref = oracle.dstedc_dc_br(d, e)
    assert rel_err(w, ref) < 1e-12


def test_nearly_scalar(solver):
    n = 20000
    rng = np.random.default_rng(5)
    d = np.full(n, 3.0)
    e = 1e-14 * rng.uniform(-1.0, 1.0, n - 1)
    w = solve(solver, d, e)
    ref = oracle.dstedc_dc_br(d, e)
    assert rel_err(w, ref) < 1e-12


@pytest.mark.parametrize("scale", [1e-150, 1e150])
def test_adjoint_under_scaling(solver, scale):
    """dL/dD and dL/dE of sum g_i lambda_i are invariant under scaling of
    the matrix (lambda is homogeneous of degree one)."""
    import torch

    n = 800
    d, e = families.generate("normal", n)
    g = torch.tensor(np.random.default_rng(2).standard_normal(n), device="cuda")
    a = solver.dstebr_backward(torch.tensor(d, device="cuda"), torch.tensor(e, device="cuda"), g)
    b = solver.dstebr_backward(torch.tensor(d * scale, device="cuda"),
                               torch.tensor(e * scale, device="cuda"), g)
    for x, y in zip(a, b):
        x, y = x.cpu().numpy(), y.cpu().numpy()
        assert np.all(np.isfinite(y))
        assert np.max(np.abs(x - y)) < 1e-10 * np.max(np.abs(x))
