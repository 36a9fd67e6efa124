"""Time the reference CUDA prototype's values-only solve on this GPU --
BENCHMARK INFRASTRUCTURE ONLY (the product never calls it).

    python oracle/time_ref_gpu.py [family] [n] [solves]

Runs ``tridiag_solver_run_from_device_tridiagonal`` (gpu/src/tridiag_solver.cu:2541),
built from the reference's sources by ``oracle/build_ref.sh`` into
``oracle/_ref/``, on the seeded instance of the given family and order
(defaults: uniform, 65536, 5), and prints one JSON line: median and
minimum ms per solve from CUDA events on the prototype's own stream, its
workspace bytes, and its max error against LAPACK DSTERF over ||T||.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(HERE, "..", "ppopp27-brdc-ae_b200"))


def main() -> None:
    import scipy.linalg.lapack as la
    import torch

    import ref_gpu
    from brdc import families

    fam = sys.argv[1] if len(sys.argv) > 1 else "uniform"
    n = int(sys.argv[2]) if len(sys.argv) > 2 else 65536
    solves = int(sys.argv[3]) if len(sys.argv) > 3 else 5
    d, e = families.generate(fam, n)
    R = ref_gpu.RefSolver()
    D = torch.tensor(d, device="cuda")
    E = torch.tensor(e, device="cuda")
    W = torch.empty(n, dtype=torch.float64, device="cuda")
    with torch.cuda.stream(R.stream):
        R.solve(D, E, W)  # warm-up
        R.stream.synchronize()
        times = []
        for _ in range(solves):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(R.stream)
            R.solve(D, E, W)
            e1.record(R.stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    w = np.sort(W.cpu().numpy())
    ref, info = la.dsterf(d.copy(), e.copy())
    ref = np.sort(ref)
    print(json.dumps({
        "impl": "reference CUDA prototype", "family": fam, "n": n, "solves": solves,
        "ms_median": float(np.median(times)), "ms_min": float(np.min(times)),
        "workspace_bytes": ref_gpu.workspace_size(n),
        "max_err_vs_dsterf": float(np.max(np.abs(w - ref)) / np.max(np.abs(ref))),
    }))
    R.close()


if __name__ == "__main__":
    main()
