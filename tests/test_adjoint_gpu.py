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


def test_autograd_two_matrices_of_one_order_in_one_loss(solver):
    """Two forwards of the same order before one backward: each backward
    must read its own forward's checkpoints."""
    import torch

    from brdc.autograd import eigvalsh_tridiagonal

    n = 800
    mats = [families.generate("normal", n, instance=s) for s in (11, 12)]
    rng = np.random.default_rng(5)
    gs = [rng.standard_normal(n) for _ in mats]
    leaves = []
    loss = 0.0
    for (d, e), g in zip(mats, gs):
        D = torch.tensor(d, device="cuda", requires_grad=True)
        E = torch.tensor(e, device="cuda", requires_grad=True)
        leaves.append((D, E))
        loss = loss + (eigvalsh_tridiagonal(D, E, solver) * torch.tensor(g, device="cuda")).sum()
    loss.backward()
    for (d, e), g, (D, E) in zip(mats, gs, leaves):
        rd, re = eig_ref_grads(d, e, g)
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


def test_central_differences_normal_n512(solver):
    """Central differences with h = 1e-6 ||T|| on the normal family at
    N = 512.  Where the spectrum has a gap near h (this instance's smallest
    is 4e-6) the difference quotient itself is off by O(1); each entry is
    therefore checked against its own truncation estimate, the Richardson
    difference |FD(2h) - FD(h)| (the O(h^2) error of FD(h) is a third of
    it), besides a floor of 1e-6 of the gradient's scale."""
    import torch

    n = 512
    d, e = families.generate("normal", n)
    rng = np.random.Generator(np.random.PCG64([2, n, 1]))
    g = rng.standard_normal(n)
    gd, ge = grads(solver, d, e, g)
    h = 1e-6 * float(np.max(np.abs(scipy.linalg.eigvalsh_tridiagonal(d, e))))
    Gt = torch.tensor(g, device="cuda")

    def loss(dd, ee):
        W = solver.dstebr(torch.tensor(dd, device="cuda"), torch.tensor(ee, device="cuda"))
        return float((W * Gt).sum())

    def fd_pair(base, j, other, first):
        v = {}
        for k in (2, 1, -1, -2):
            p = base.copy()
            p[j] += k * h
            v[k] = loss(p, other) if first else loss(other, p)
        return (v[1] - v[-1]) / (2 * h), (v[2] - v[-2]) / (4 * h)

    sc = max(np.max(np.abs(gd)), np.max(np.abs(ge)))
    resolved = 0
    for ours, base, other, first in ((gd, d, e, True), (ge, e, d, False)):
        for j in range(base.shape[0]):
            f1, f2 = fd_pair(base, j, other, first)
            bound = 1e-6 * sc + 2.0 * abs(f2 - f1)
            assert abs(ours[j] - f1) < bound, (first, j, ours[j], f1, f2)
            resolved += abs(f2 - f1) < 1e-6 * sc
    # the estimate only widens the bar where FD cannot resolve the gradient
    assert resolved > 0.95 * (2 * n - 1)


def test_batched_backward_matches_single(solver):
    """The batched adjoint equals the single-instance adjoint of every
    instance (to the parity tolerance: lanes per root follow the batch's K
    statistics) and the LAPACK eigenvector gradient."""
    import torch

    off, D, E, orders, fams = families.batch(24, 17, 1500, seed=5)
    rng = np.random.default_rng(11)
    G = rng.standard_normal(off[-1])
    Dt, Et, Gt = (torch.tensor(x, device="cuda") for x in (D, E, G))
    gD, gE = solver.dstebr_batched_backward(off, Dt, Et, Gt)
    gD, gE = gD.cpu().numpy(), gE.cpu().numpy()
    for b in range(len(orders)):
        lo, hi = int(off[b]), int(off[b + 1])
        d, e, g = D[lo:hi], E[lo:hi - 1], G[lo:hi]
        sd, se = grads(solver, d, e, g)
        rd, re = eig_ref_grads(d, e, g)
        sc = max(np.max(np.abs(rd)), np.max(np.abs(re)), 1e-300)
        # clustered spectra (gaps ~1e-13) amplify rounding differences and
        # defeat double-precision eigenvectors; see the multiprecision test
        tol = 1e-6 if fams[b] == "clustered" else 1e-11
        assert np.max(np.abs(gD[lo:hi] - sd)) < tol * sc, b
        assert np.max(np.abs(gE[lo:hi - 1] - se)) < tol * sc, b
        if fams[b] != "clustered":
            assert np.max(np.abs(gD[lo:hi] - rd)) < 1e-9 * sc, b
            assert np.max(np.abs(gE[lo:hi - 1] - re)) < 1e-9 * sc, b
        assert gE[hi - 1] == 0.0


def test_batched_backward_keep_forward(solver):
    import torch

    off, D, E, orders, _ = families.batch(16, 40, 900, seed=6)
    G = np.random.default_rng(12).standard_normal(off[-1])
    Dt, Et, Gt = (torch.tensor(x, device="cuda") for x in (D, E, G))
    ws = solver.batched_workspace(off, checkpoints=True)
    W = solver.dstebr_batched(off, Dt, Et, workspace=ws)
    a1, b1 = solver.dstebr_batched_backward(off, Dt, Et, Gt, workspace=ws, keep_forward=True)
    a2, b2 = solver.dstebr_batched_backward(off, Dt, Et, Gt, workspace=ws, keep_forward=False)
    assert torch.equal(a1, a2) and torch.equal(b1, b2)
    W2 = solver.dstebr_batched(off, Dt, Et)
    assert torch.equal(W, W2)


@pytest.mark.parametrize("family,n", [("uniform", 20000), ("toeplitz", 6000), ("normal", 12000)])
def test_fused_levels_same_gradient(solver, family, n):
    """The checkpoint a fused-level solve leaves (merges finished by k_level,
    big ones by the sweep kernel) serves the adjoint like the per-level one."""
    import brdc

    d, e = families.generate(family, n)
    g = np.random.default_rng(11).standard_normal(n)
    s = brdc.Solver()
    try:
        out = []
        for fuse in (0, 1 << 30):
            s.set_tuning(fused_level_rows=fuse)
            out.append(grads(s, d, e, g))
        sc = max(np.max(np.abs(out[0][0])), np.max(np.abs(out[0][1])))
        assert np.max(np.abs(out[1][0] - out[0][0])) < 1e-11 * sc
        assert np.max(np.abs(out[1][1] - out[0][1])) < 1e-11 * sc
    finally:
        s.close()
