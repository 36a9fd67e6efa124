"""Parity of the sm_100a solve with the oracle (C restatement of the
reference's DSTEDC_DC_BR), LAPACK DSTERF and closed forms."""
import json
import os

import numpy as np
import pytest

import oracle
from brdc import families

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-12  # max |lambda - lambda_ref| / ||T||_2


def gpu_solve(solver, d, e):
    import torch

    D = torch.tensor(d, dtype=torch.float64, device="cuda")
    E = torch.tensor(e if len(e) else np.zeros(1), dtype=torch.float64, device="cuda")
    W = solver.dstebr(D, E)
    info = solver.info(len(d))
    assert info == 0, f"info={info}"
    return W.cpu().numpy()


def rel_err(w, ref):
    return float(np.max(np.abs(w - ref)) / max(np.max(np.abs(ref)), 1e-300))


@pytest.mark.parametrize("n", list(range(1, 70)))
def test_small_orders_every_tree_shape(solver, n):
    rng = np.random.default_rng(1000 + n)
    d, e = rng.standard_normal(n), rng.standard_normal(max(n - 1, 0))
    w = gpu_solve(solver, d, e)
    assert np.all(np.diff(w) >= 0)
    assert rel_err(w, np.sort(oracle.dsterf(d, e))) < TOL


@pytest.mark.parametrize("family", ["uniform", "normal", "clustered"])
@pytest.mark.parametrize("n", [100, 1000, 4096, 8192])
def test_families_vs_oracle(solver, family, n):
    d, e = families.generate(family, n)
    w = gpu_solve(solver, d, e)
    ref = oracle.dstedc_dc_br(d, e)
    assert rel_err(w, ref) < TOL
    assert rel_err(w, np.sort(oracle.dsterf(d, e))) < TOL


@pytest.mark.parametrize("n", [17, 33, 100, 4096, 65536])
def test_toeplitz_closed_form(solver, n):
    d, e = families.generate("toeplitz", n)
    assert rel_err(gpu_solve(solver, d, e), families.toeplitz_eigenvalues(n)) < TOL


@pytest.mark.parametrize("family", ["uniform", "normal", "clustered"])
def test_full_size_vs_oracle(solver, family):
    d, e = families.generate(family, 65536)
    assert rel_err(gpu_solve(solver, d, e), oracle.dstedc_dc_br(d, e)) < TOL


def test_reference_fixture_slice(solver):
    z = np.load(os.path.join(GOLDEN, "reduced_dense_lead4096.npz"))
    assert rel_err(gpu_solve(solver, z["d"], z["e"]), z["dsterf"]) < TOL


def test_sign_of_offdiagonal_ignored(solver):
    d, e = families.generate("normal", 3000)
    w1 = gpu_solve(solver, d, e)
    w2 = gpu_solve(solver, d, -e)
    w3 = gpu_solve(solver, d, np.abs(e))
    assert np.array_equal(w1, w2) and np.array_equal(w1, w3)


def test_zero_couplings_block_diagonal(solver):
    rng = np.random.default_rng(5)
    d, e = rng.standard_normal(2048), rng.standard_normal(2047)
    e[::37] = 0.0
    e[1023] = 0.0  # the root cut
    assert rel_err(gpu_solve(solver, d, e), np.sort(oracle.dsterf(d, e))) < TOL


def test_diagonal_matrix(solver):
    rng = np.random.default_rng(6)
    d = rng.standard_normal(1000)
    assert np.array_equal(gpu_solve(solver, d, np.zeros(999)), np.sort(d))


def test_repeated_solves_bitwise_stable(solver):
    d, e = families.generate("uniform", 20000)
    w1 = gpu_solve(solver, d, e)
    w2 = gpu_solve(solver, d, e)
    assert np.array_equal(w1, w2)


def test_trace_and_frobenius(solver):
    d, e = families.generate("normal", 65536)
    w = gpu_solve(solver, d, e)
    assert abs(w.sum() - d.sum()) < 1e-10 * np.abs(w).sum()
    assert abs((w * w).sum() - (d * d).sum() - 2 * (e * e).sum()) < 1e-10 * (w * w).sum()


def test_diagnostics_counts(solver):
    d, e = families.generate("uniform", 4096)
    gpu_solve(solver, d, e)
    dg = solver.diagnostics(4096)
    assert dg["levels"] == 8 and dg["leaf_count"] == 256
    for k, lv in enumerate(dg["level"]):
        assert lv["merge_count"] == 2 ** (7 - k)
        assert lv["size_sum"] == 4096
        assert 0 <= lv["dd_after_sum"] <= lv["dd_before_sum"] <= 4096
        assert lv["secular_iter_failed"] == 0


def test_lapack_style_host_entry(built_lib):
    import brdc

    d, e = families.generate("normal", 5000)
    w = brdc.dstedc_dc_br(d, e)
    assert rel_err(w, np.sort(oracle.dsterf(d, e))) < TOL


@pytest.mark.parametrize("family,n", [("uniform", 20000), ("toeplitz", 5000), ("clustered", 9000)])
def test_tunings_agree(solver, family, n):
    """Launch shapes do not change what is computed: the same deflation
    counts at every level and the same eigenvalues to rounding, whatever
    the subtree depth, deflation cluster, sweep parallelism and level
    fusion."""
    import torch

    import brdc

    d, e = families.generate(family, n)
    D = torch.tensor(d, device="cuda")
    E = torch.tensor(e, device="cuda")
    s = brdc.Solver()
    ref_w, ref_k = None, None
    try:
        ws = s.workspace(n)
        for sub in (-1, 0, 1, 2, 3, 4, 5):
            for cl in (1, 16):
                for lanes in (8192, 75776, 1 << 20):
                    for fuse in (0, 4096, 1 << 30):
                        s.set_tuning(subtree_levels=sub, deflate_cluster=cl,
                                     sweep_lanes_target=lanes, fused_level_rows=fuse)
                        W = s.dstebr(D, E, workspace=ws).cpu().numpy()
                        K = [lv["dd_after_sum"] for lv in s.diagnostics(n, ws)["level"]]
                        if ref_w is None:
                            ref_w, ref_k = W, K
                            continue
                        key = (sub, cl, lanes, fuse)
                        assert K == ref_k, key
                        err = np.max(np.abs(W - ref_w)) / np.max(np.abs(ref_w))
                        assert err < 1e-13, (key, err)
    finally:
        s.close()


def test_tuning_validation(solver):
    import brdc

    s = brdc.Solver()
    try:
        for bad in ({"subtree_levels": 6}, {"deflate_cluster": 3}, {"sweep_lanes_target": 10},
                    {"fused_level_rows": -1}):
            with pytest.raises(brdc.BrdcError):
                s.set_tuning(**bad)
        s.set_tuning(subtree_levels=2, deflate_cluster=4, sweep_lanes_target=50000,
                     fused_level_rows=8192)
        assert s.tuning() == {"subtree_levels": 2, "deflate_cluster": 4,
                              "sweep_lanes_target": 50000, "fused_level_rows": 8192}
    finally:
        s.close()


def test_default_tuning(solver):
    """A new handle carries the documented default launch shapes."""
    import brdc

    s = brdc.Solver()
    try:
        assert s.tuning() == {"subtree_levels": -1, "deflate_cluster": 16,
                              "sweep_lanes_target": 303104, "fused_level_rows": 1 << 30}
    finally:
        s.close()


def test_autotune_single_and_batched(solver):
    """The autotuner leaves a valid tuning on the handle, and solves under it
    stay correct."""
    import torch

    import brdc

    s = brdc.Solver()
    try:
        n = 20000
        d, e = families.generate("normal", n)
        D = torch.tensor(d, device="cuda")
        E = torch.tensor(e, device="cuda")
        t = s.autotune(D, E)
        assert t == s.tuning()
        assert -1 <= t["subtree_levels"] <= 5 and t["deflate_cluster"] in (1, 2, 4, 8, 16)
        W = s.dstebr(D, E).cpu().numpy()
        ref = oracle.dstedc_dc_br(d, e)
        assert np.max(np.abs(W - ref)) / np.max(np.abs(ref)) < 1e-12

        off, Db, Eb, orders, _ = families.batch(40, 17, 2500, seed=8)
        Dt = torch.tensor(Db, device="cuda")
        Et = torch.tensor(Eb, device="cuda")
        tb = s.autotune(Dt, Et, offsets=off)
        assert tb == s.tuning()
        Wb = s.dstebr_batched(off, Dt, Et).cpu().numpy()
        for b in range(len(orders)):
            lo, hi = int(off[b]), int(off[b + 1])
            ref = oracle.dstedc_dc_br(Db[lo:hi], Eb[lo:hi - 1])
            assert np.max(np.abs(Wb[lo:hi] - ref)) / np.max(np.abs(ref)) < 1e-12
    finally:
        s.close()
