"""The eigenvector path (brdc_dstebr_vectors): orthogonality and residual of
the eigenvectors, eigenvalues identical to the values-only solve, against
LAPACK's eigenvectors where the spectrum is well separated."""
import numpy as np
import pytest

import oracle
from brdc import families

pytestmark = pytest.mark.gpu


def tri_matvec(d, e, Z):
    """T Z for the symmetric tridiagonal T = (d, e)."""
    TZ = d[:, None] * Z
    if len(e):
        TZ[:-1] += e[:, None] * Z[1:]
        TZ[1:] += e[:, None] * Z[:-1]
    return TZ


def check(solver, d, e, tol_orth, tol_res):
    import torch

    n = len(d)
    D = torch.tensor(d, device="cuda")
    E = torch.tensor(e if n > 1 else np.zeros(1), device="cuda")
    W, Z = solver.dstebr_vectors(D, E)
    w = W.cpu().numpy()
    z = Z.cpu().numpy()
    assert np.all(np.diff(w) >= 0)
    # the eigenvalues are those of the values-only solve, bit for bit
    assert np.array_equal(w, solver.dstebr(D, E).cpu().numpy())
    norm = max(np.max(np.abs(w)), 1e-300)
    orth = np.max(np.abs(z.T @ z - np.eye(n)))
    res = np.max(np.abs(tri_matvec(d, e, z) - z * w[None, :])) / norm
    assert orth < tol_orth, orth
    assert res < tol_res, res
    return w, z, orth, res


@pytest.mark.parametrize("n", [1, 2, 5, 16, 17, 31, 33, 100, 257, 1000])
def test_small_orders(solver, n):
    rng = np.random.default_rng(500 + n)
    d, e = rng.standard_normal(n), rng.standard_normal(max(n - 1, 0))
    check(solver, d, e, 1e-12, 1e-13)


@pytest.mark.parametrize("family", ["uniform", "normal", "clustered", "toeplitz"])
@pytest.mark.parametrize("n", [2048, 4096])
def test_families(solver, family, n):
    d, e = families.generate(family, n)
    w, _, _, _ = check(solver, d, e, 1e-11, 1e-12)
    assert np.max(np.abs(w - np.sort(oracle.dsterf(d, e)))) < 1e-12 * np.max(np.abs(w))


def test_against_lapack_vectors(solver):
    # separated spectrum: each eigenvector is determined up to sign
    import scipy.linalg

    n = 600
    d = np.arange(n, dtype=np.float64) + 0.1 * np.sin(np.arange(n))
    e = 0.3 * np.cos(np.arange(n - 1))
    _, z, _, _ = check(solver, d, e, 1e-12, 1e-13)
    wl, zl = scipy.linalg.eigh_tridiagonal(d, e)
    dots = np.abs(np.sum(z * zl, axis=0))
    assert np.max(np.abs(dots - 1.0)) < 1e-10


def test_zero_and_negative_couplings(solver):
    rng = np.random.default_rng(77)
    n = 700
    d = rng.standard_normal(n)
    e = rng.standard_normal(n - 1)
    e[::37] = 0.0
    e[5::11] *= -1.0
    check(solver, d, e, 1e-12, 1e-13)


@pytest.mark.parametrize("n", [3001, 5000])
def test_two_node_sizes(solver, n):
    # orders that are not powers of two: every level has nodes of two sizes,
    # hence four GEMM shapes
    d, e = families.generate("normal", n)
    check(solver, d, e, 1e-11, 1e-12)


def test_graph_capture(solver):
    import ctypes

    import torch

    import brdc

    n = 3001
    d, e = families.generate("uniform", n)
    D = torch.tensor(d, device="cuda")
    E = torch.tensor(e, device="cuda")
    s = brdc.Solver()
    g = None
    try:
        nb = ctypes.c_size_t(0)
        brdc.load().brdc_dstebr_vectors_workspace_size(n, ctypes.byref(nb))
        ws = torch.empty(nb.value, dtype=torch.uint8, device="cuda")
        stream = torch.cuda.Stream()
        stream.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(stream):
            s.set_stream(stream)
            W0, Z0 = s.dstebr_vectors(D, E, workspace=ws)  # outside the capture first
            W0, Z0 = W0.clone(), Z0.clone()
            stream.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=stream):
                W1, Z1 = s.dstebr_vectors(D, E, workspace=ws)
            g.replay()
            stream.synchronize()
        # captured, M is laid out by each level's largest node (nothing can
        # be read back); the products still take each node's own columns and
        # surviving rows: the same vectors bit for bit
        assert torch.equal(W0, W1)
        assert torch.equal(Z0, Z1)
    finally:
        del g
        s.set_stream(torch.cuda.current_stream())
        s.close()
