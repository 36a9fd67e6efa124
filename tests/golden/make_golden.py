"""Regenerate the committed golden fixtures (run in the build container,
where the reference tree is readable):

    python tests/golden/make_golden.py /root/reference

The reference ships one input fixture and no expected eigenvalues:
data/inputs/reduced_dense_49152.de.bin (int64 n, then n D doubles and n-1 E
doubles; format of gpu/bench/tridiag_dc_bench.cu:393-427).  This script
stores a small slice of it (the leading 4096 x 4096 principal tridiagonal)
together with LAPACK DSTERF eigenvalues of that slice, plus summary values
of the full 49,152 problem (input CRC, trace, DSTERF spectrum moments and
extremes, and the oracle's max deviation from DSTERF), so the tests can pin
the oracle and the GPU solver on the reference's own data without the
reference tree being present.
"""
import json
import os
import sys
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle  # noqa: E402

LEAD = 4096


def main(ref_root: str) -> None:
    path = os.path.join(ref_root, "data", "inputs", "reduced_dense_49152.de.bin")
    raw = open(path, "rb").read()
    n = int(np.frombuffer(raw[:8], dtype=np.int64)[0])
    d = np.frombuffer(raw[8:8 + 8 * n], dtype=np.float64).copy()
    e = np.frombuffer(raw[8 + 8 * n:], dtype=np.float64).copy()
    assert e.shape[0] == n - 1, (n, e.shape)
    w_full = np.sort(oracle.dsterf(d, e))
    w_br = oracle.dstedc_dc_br(d, e)
    scale = float(np.max(np.abs(w_full)))
    summary = {
        "source": "data/inputs/reduced_dense_49152.de.bin",
        "n": n,
        "crc32": zlib.crc32(raw),
        "negative_e": int(np.sum(e < 0)),
        "trace": float(np.sum(d)),
        "frobenius2": float(np.sum(d * d) + 2.0 * np.sum(e * e)),
        "dsterf_min": float(w_full[0]),
        "dsterf_max": float(w_full[-1]),
        "dsterf_sum": float(np.sum(w_full)),
        "dsterf_sumsq": float(np.sum(w_full * w_full)),
        "oracle_vs_dsterf_max_rel": float(np.max(np.abs(w_br - w_full)) / scale),
        "lead": LEAD,
    }
    dl, el = d[:LEAD].copy(), e[:LEAD - 1].copy()
    wl = np.sort(oracle.dsterf(dl, el))
    np.savez_compressed(os.path.join(HERE, "reduced_dense_lead4096.npz"), d=dl, e=el, dsterf=wl)
    with open(os.path.join(HERE, "reduced_dense_49152_summary.json"), "w") as f:
        json.dump(summary, f, indent=1, sort_keys=True)
    print(json.dumps(summary, indent=1))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
