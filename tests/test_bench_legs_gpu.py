"""The bench's multi-GPU batch leg and reference-comparison leg run on one
GPU too (world size 1): the sharded batch solves every instance of
config 3 and reports a rate; the cuSOLVER probe reports what it found."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench_mod(built_lib):
    sys.path.insert(0, ROOT)
    import bench

    return bench


def test_sharded_batch_leg_on_one_rank(bench_mod):
    import torch

    import brdc
    from brdc import families

    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    out = bench_mod.bench_sharded_batch(torch, brdc, families, 0, 1, None, flush)
    assert out["count"] == 4096 and out["ranks"] == 1
    assert out["info_rank0"] == 0
    assert out["ms"] > 0 and np.isfinite(out["solves_per_s"])
    assert abs(out["balance_sum_n2_max_over_mean"] - 1.0) < 1e-12


def test_xstedc_probe_reports(bench_mod):
    out = bench_mod.xstedc_probe()
    assert isinstance(out["available"], bool)
    if not out["available"]:
        assert "unavailable on this box" in out["note"]
