"""Adjoint of the BR solve: dL/dD, dL/dE for L = sum g_i lambda_i against
central finite differences (N=512) and against the LAPACK eigenvector
gradient sum_i g_i v_ij^2, 2 sum_i g_i v_ij v_i,j+1 (N=4096)."""
import os

import numpy as np
import pytest
import scipy.linalg

from brdc import families

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def grads(solver, d, e, g):
    import torch

    D = torch.tensor(d, device="cuda")
    E = torch.tensor(e, device="cuda")
    G = torch.tensor(g, device="cuda")
    gD, gE = solver.dstebr_backward(D, E, G)
    return gD.cpu().numpy(), gE.cpu().numpy()


def eig_ref_grads(d, e, g):
    w, V = scipy.linalg.eigh_tridiagonal(d, e)
    gd = (V * V) @ g
    ge = 2.0 * (V[:-1] * V[1:]) @ g
    return gd, ge


@pytest.mark.parametrize("n", [17, 40, 100, 300])
def test_small_orders_vs_eigenvectors(solver, n):
    rng = np.random.default_rng(100 + n)
    d, e = rng.standard_normal(n), rng.standard_normal(n - 1)
    g = rng.standard_normal(n)
    gd, ge = grads(solver, d, e, g)
    rd, re = eig_ref_grads(d, e, g)
    sc = max(np.max(np.abs(rd)), np.max(np.abs(re)))
    assert np.max(np.abs(gd - rd)) < 1e-9 * sc
    assert np.max(np.abs(ge - re)) < 1e-9 * sc


def test_finite_differences_n512(solver):
    """Fourth-order central differences of L = sum g_i lambda_i, one entry
    of D or E at a time.  The matrix is a strongly coupled random
    tridiagonal (d ~ 0.1 N(0,1), e ~ 1 + 0.1 N(0,1)): its eigenvectors are
    extended, so its smallest eigenvalue gap (~8e-5) is far above the step.
    Random diagonals with localized eigenvectors have gaps near 1e-6, where
    the gradient turns over within one step and no difference quotient
    resolves it (LAPACK's own eigenvalues fail the same check there)."""
    import torch

    n = 512
    rng = np.random.Generator(np.random.PCG64([11, n, 0]))
    d = 0.1 * rng.standard_normal(n)
    e = 1.0 + 0.1 * rng.standard_normal(n - 1)
    g = rng.standard_normal(n)
    gd, ge = grads(solver, d, e, g)
    scale = float(np.max(np.abs(scipy.linalg.eigvalsh_tridiagonal(d, e))))
    h = 1e-5 * scale
    Gt = torch.tensor(g, device="cuda")

    def loss(dd, ee):
        W = solver.dstebr(torch.tensor(dd, device="cuda"), torch.tensor(ee, device="cuda"))
        return float((W * Gt).sum())

    def fd(base, j, other, first):
        v = []
        for k in (2, 1, -1, -2):
            p = base.copy()
            p[j] += k * h
            v.append(loss(p, other) if first else loss(other, p))
        return (-v[0] + 8.0 * v[1] - 8.0 * v[2] + v[3]) / (12.0 * h)

    fd_d = np.array([fd(d, j, e, True) for j in range(n)])
    fd_e = np.array([fd(e, j, d, False) for j in range(n - 1)])
    sc = max(np.max(np.abs(gd)), np.max(np.abs(ge)))
    assert np.max(np.abs(gd - fd_d)) < 1e-6 * sc
    assert np.max(np.abs(ge - fd_e)) < 1e-6 * sc


def test_lapack_eigenvector_gradient_n4096(solver):
    n = 4096
    d, e = families.generate("normal", n)
    rng = np.random.Generator(np.random.PCG64([2, n, 1]))
    g = rng.standard_normal(n)
    gd, ge = grads(solver, d, e, g)
    rd, re = eig_ref_grads(d, e, g)
    sc = max(np.max(np.abs(rd)), np.max(np.abs(re)))
    assert np.max(np.abs(gd - rd)) < 1e-9 * sc
    assert np.max(np.abs(ge - re)) < 1e-9 * sc


@pytest.mark.parametrize("family", ["uniform", "toeplitz"])
def test_other_families_vs_eigenvectors(solver, family):
    """Toeplitz (d = 2, e = 1) splits into identical children at every inner
    merge, so every pole ties with one from the other child and is rotated
    out: this pins the tie terms of the adjoint."""
    n = 2048
    d, e = families.generate(family, n)
    rng = np.random.default_rng(7)
    g = rng.standard_normal(n)
    gd, ge = grads(solver, d, e, g)
    rd, re = eig_ref_grads(d, e, g)
    sc = max(np.max(np.abs(rd)), np.max(np.abs(re)))
    assert np.max(np.abs(gd - rd)) < 1e-9 * sc
    assert np.max(np.abs(ge - re)) < 1e-9 * sc


@pytest.mark.parametrize("n", [32, 96])
def test_clustered_vs_multiprecision(solver, n):
    """Clustered spectra (8 centres, 1e-10 spread, couplings ~1e-6) have
    eigenvalue gaps down to 1e-13; the reference gradients come from
    50-digit eigenvectors (tests/golden/make_adjoint_golden.py)."""
    ref = np.load(os.path.join(GOLDEN, "adjoint_clustered.npz"))
    d, e = families.generate("clustered", n)
    g = ref[f"g{n}"]
    gd, ge = grads(solver, d, e, g)
    rd, re = ref[f"gd{n}"], ref[f"ge{n}"]
    sc = max(np.max(np.abs(rd)), np.max(np.abs(re)))
    assert np.max(np.abs(gd - rd)) < 1e-7 * sc
    assert np.max(np.abs(ge - re)) < 1e-9 * sc


def test_clustered_n2048_vs_lapack(solver):
    """At n = 2048 only double-precision eigenvectors are at hand; their own
    error on these gaps is ~1e-6 of the gradient's scale (measured against
    50-digit eigenvectors at n = 32, 96: LAPACK 3e-7 and 1e-7, this solver
    2e-8 and 3e-9)."""
    n = 2048
    d, e = families.generate("clustered", n)
    g = np.random.default_rng(7).standard_normal(n)
    gd, ge = grads(solver, d, e, g)
    rd, re = eig_ref_grads(d, e, g)
    sc = max(np.max(np.abs(rd)), np.max(np.abs(re)))
    assert np.max(np.abs(gd - rd)) < 2e-5 * sc
    assert np.max(np.abs(ge - re)) < 1e-8 * sc


def test_autograd_function(solver):
    import torch

    from brdc.autograd import eigvalsh_tridiagonal

    n = 1000
    d, e = families.generate("normal", n)
    D = torch.tensor(d, device="cuda", requires_grad=True)
    E = torch.tensor(e, device="cuda", requires_grad=True)
    W = eigvalsh_tridiagonal(D, E, solver)
    rng = np.random.default_rng(3)
    g = torch.tensor(rng.standard_normal(n), device="cuda")
    (W * g).sum().backward()
    rd, re = eig_ref_grads(d, e, g.cpu().numpy())
    sc = max(np.max(np.abs(rd)), np.max(np.abs(re)))
    assert np.max(np.abs(D.grad.cpu().numpy() - rd)) < 1e-9 * sc
    assert np.max(np.abs(E.grad.cpu().numpy() - re)) < 1e-9 * sc


def test_keep_forward_matches_rerun(solver):
    import torch

    n = 3000
    d, e = families.generate("uniform", n)
    D = torch.tensor(d, device="cuda")
    E = torch.tensor(e, device="cuda")
    G = torch.tensor(np.random.default_rng(4).standard_normal(n), device="cuda")
    ws = solver.checkpoint_workspace(n)
    solver.dstebr(D, E, workspace=ws)
    a1, b1 = solver.dstebr_backward(D, E, G, workspace=ws, keep_forward=True)
    a2, b2 = solver.dstebr_backward(D, E, G, workspace=ws, keep_forward=False)
    assert torch.equal(a1, a2) and torch.equal(b1, b2)
