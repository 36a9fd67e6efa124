"""The reference's own inputs through the sm_100a solve: the GPU bench's data
modes (gpu/bench/tridiag_dc_bench.cu:229-339), the DLATMS spectrum-prescribed
matrices of the paper's figures (cpu/jobs/run_spectrum_de_cache_job.sh:52-110,
whose prescribed spectrum is the exact answer) and a .de.bin round trip."""
import numpy as np
import pytest

import oracle
from brdc import families, inputs

pytestmark = pytest.mark.gpu
TOL = 1e-12  # max |lambda - lambda_ref| / ||T||_2


def gpu_solve(solver, d, e):
    import torch

    D = torch.tensor(d, dtype=torch.float64, device="cuda")
    E = torch.tensor(e if len(e) else np.zeros(1), dtype=torch.float64, device="cuda")
    W = solver.dstebr(D, E)
    assert solver.info(len(d)) == 0
    return W.cpu().numpy()


def rel_err(w, ref):
    return float(np.max(np.abs(w - ref)) / max(np.max(np.abs(ref)), 1e-300))


@pytest.mark.parametrize("mode", inputs.GPU_BENCH_MODES)
@pytest.mark.parametrize("n", [17, 1000, 4096])
def test_gpu_bench_modes(solver, mode, n):
    if mode == "test" and n > 1000:
        pytest.skip("the test mode draws n^2 numbers; 1000 is enough")
    d, e = inputs.generate(mode, n, index=1)
    w = gpu_solve(solver, d, e)
    assert rel_err(w, oracle.dstedc_dc_br(d, e)) < TOL
    assert rel_err(w, np.sort(oracle.dsterf(d, e))) < TOL
    if mode == "toeplitz":
        assert rel_err(w, families.toeplitz_eigenvalues(n, 2.0, 0.25)) < TOL


@pytest.mark.parametrize("mode", ["uniform", "normal", "clustered"])
@pytest.mark.parametrize("n", [600, 4096])
def test_spectrum_prescribed(solver, mode, n):
    d, e, info, eig = inputs.spectrum_case(mode, n)
    assert info == 0
    w = gpu_solve(solver, d, e)
    assert rel_err(w, np.sort(eig)) < TOL
    assert rel_err(w, oracle.dstedc_dc_br(d, e)) < TOL


def test_de_file_roundtrip_solve(solver, tmp_path):
    d, e = inputs.generate("normal", 3000)
    p = str(tmp_path / "normal_3000.de.bin")
    inputs.write_de(p, d, e)
    d2, e2 = inputs.read_de(p)
    assert np.array_equal(gpu_solve(solver, d2, e2), gpu_solve(solver, d, e))
