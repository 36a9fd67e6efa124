"""The oracle (C restatement of DSTEDC_DC_BR) pinned against LAPACK DSTERF,
closed-form spectra and the reference's own data fixture."""
import json
import os

import numpy as np
import pytest

import oracle
from brdc import families

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel_err(w, ref):
    return float(np.max(np.abs(np.asarray(w) - np.asarray(ref))) / max(np.max(np.abs(ref)), 1e-300))


def test_smoke_semantics_uniform_pm1():
    # scripts/cpu/smoke_br.f90:19-38: U(-1,1) D and E, N=4096, BR vs DSTERF
    # max |d-w| / max|w| < 1e-10 (README: ~1e-14 observed)
    rng = np.random.default_rng(20240)
    d = rng.uniform(-1, 1, 4096)
    e = rng.uniform(-1, 1, 4095)
    assert rel_err(oracle.dstedc_dc_br(d, e), np.sort(oracle.dsterf(d, e))) < 1e-12


@pytest.mark.parametrize("family", ["uniform", "normal", "clustered"])
def test_families_vs_dsterf(family):
    d, e = families.generate(family, 4096)
    assert rel_err(oracle.dstedc_dc_br(d, e), np.sort(oracle.dsterf(d, e))) < 1e-12


@pytest.mark.parametrize("n", [26, 100, 1000, 4096])
def test_toeplitz_closed_form(n):
    d, e = families.generate("toeplitz", n)
    assert rel_err(oracle.dstedc_dc_br(d, e), families.toeplitz_eigenvalues(n)) < 1e-13


@pytest.mark.parametrize("n", list(range(1, 40)) + [64, 65, 127, 128, 129])
def test_small_orders(n):
    rng = np.random.default_rng(n)
    d, e = rng.standard_normal(n), rng.standard_normal(max(n - 1, 0))
    assert rel_err(oracle.dstedc_dc_br(d, e), np.sort(oracle.dsterf(d, e))) < 1e-13


def test_negligible_offdiagonals_split():
    # dstedc_dc_br.f:94-111 splits at |E| <= eps*sqrt|D_i|*sqrt|D_i+1|
    rng = np.random.default_rng(3)
    d, e = rng.standard_normal(300), rng.standard_normal(299)
    e[[40, 41, 150, 298]] = 0.0
    assert rel_err(oracle.dstedc_dc_br(d, e), np.sort(oracle.dsterf(d, e))) < 1e-13


def test_workspace_query_formula():
    # dstedc_dc_br.f:44-75: LWMIN=(16+2*NTHR)*N, LIWMIN=7N for N>SMLSIZ(=25)
    nthr = oracle._load().brdc_wprod_nthreads()
    assert oracle.dstedc_dc_br_query(4096) == ((16 + 2 * nthr) * 4096, 7 * 4096)
    assert oracle.dstedc_dc_br_query(25) == (1, 1)
    assert oracle.dstedc_dc_br_query(0) == (1, 1)


def test_reference_fixture_slice():
    z = np.load(os.path.join(GOLDEN, "reduced_dense_lead4096.npz"))
    assert rel_err(oracle.dstedc_dc_br(z["d"], z["e"]), z["dsterf"]) < 1e-12
    assert np.sum(z["e"] < 0) > 0  # mixed signs exercise the |E| path


def test_reference_fixture_summary():
    s = json.load(open(os.path.join(GOLDEN, "reduced_dense_49152_summary.json")))
    assert s["n"] == 49152 and s["negative_e"] == 24779
    assert s["oracle_vs_dsterf_max_rel"] < 1e-12
    # eigenvalue moments equal trace(T) and ||T||_F^2
    assert abs(s["dsterf_sum"] - s["trace"]) < 1e-12 * abs(s["trace"])
    assert abs(s["dsterf_sumsq"] - s["frobenius2"]) < 1e-12 * s["frobenius2"]


def test_deflation_log_counts():
    d, e = families.generate("normal", 4096)
    _, kd = oracle.dstedc_dc_br(d, e, return_kdefl=True)
    # 4096 = 2^8 leaves of 16 at SMLSIZ 25: 255 merges
    assert kd.shape[0] == 255
    assert np.all(kd >= 0) and np.all(kd <= 4096)
