"""Time the reference CUDA prototype's values-only solve on this GPU --
BENCHMARK INFRASTRUCTURE ONLY (the product never calls it).

    python oracle/time_ref_gpu.py [SPEC ...] [--solves S]

Runs ``tridiag_solver_run_from_device_tridiagonal`` (gpu/src/tridiag_solver.cu:2541),
built from the reference's sources by ``oracle/build_ref.sh`` into
``oracle/_ref/``, and prints one JSON line per input: median and minimum ms
per solve from CUDA events on the prototype's own stream, its workspace
bytes, and its max error over ||T||.

A SPEC is what ``bench.py --data`` takes, so both solvers can be timed on
the same data: MODE:N for the reference GPU bench's own data modes (bench,
test, normal, uniform, toeplitz, clustered), spectrum-MODE:N for the
paper's DLATMS spectrum-prescribed matrices, family-NAME:N for the seeded
families of the plain-solve configuration (uniform, normal, toeplitz,
clustered).  Default: family-uniform:65536, the headline input.

The error is against the exact spectrum where the input prescribes one
(Toeplitz closed forms, DLATMS), else against LAPACK bisection (DSTEBZ) on
64 sampled eigenvalues, extremes included.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(HERE, "..", "ppopp27-brdc-ae_b200"))


def load(spec):
    """(d, e, exact spectrum or None) of one SPEC."""
    from brdc import families, inputs

    name, _, n = spec.partition(":")
    n = int(n) if n else 65536
    if name.startswith("spectrum-"):
        d, e, info, eig = inputs.spectrum_case(name[len("spectrum-"):], n)
        if info != 0:
            raise RuntimeError(f"DLATMS info {info} for {spec}")
        exact = np.sort(eig) if eig is not None else families.toeplitz_eigenvalues(n, 2.0, 0.25)
        return d, e, exact
    if name.startswith("family-"):
        fam = name[len("family-"):]
        d, e = families.generate(fam, n)
        return d, e, families.toeplitz_eigenvalues(n) if fam == "toeplitz" else None
    d, e = inputs.generate(name, n)
    return d, e, families.toeplitz_eigenvalues(n, 2.0, 0.25) if name == "toeplitz" else None


def sampled_error(d, e, w, blocks=16, width=4):
    """max |w_i - lambda_i| / ||T|| over `blocks` runs of `width`
    consecutive eigenvalues from LAPACK bisection, the first and last
    included."""
    import scipy.linalg

    n = len(d)
    starts = np.unique(np.linspace(0, max(n - width, 0), blocks).astype(int))
    lo = scipy.linalg.eigvalsh_tridiagonal(d, e, select="i", select_range=(0, 0), lapack_driver="stebz")
    hi = scipy.linalg.eigvalsh_tridiagonal(d, e, select="i", select_range=(n - 1, n - 1),
                                           lapack_driver="stebz")
    norm = max(abs(lo[0]), abs(hi[0]))
    worst = 0.0
    for st in starts:
        top = min(st + width - 1, n - 1)
        ref = scipy.linalg.eigvalsh_tridiagonal(d, e, select="i", select_range=(int(st), int(top)),
                                                lapack_driver="stebz")
        worst = max(worst, float(np.max(np.abs(w[st:top + 1] - ref))))
    return worst / norm


def main() -> None:
    import torch

    import ref_gpu

    args = sys.argv[1:]
    solves = 5
    if "--solves" in args:
        i = args.index("--solves")
        solves = int(args[i + 1])
        del args[i:i + 2]
    specs = args or ["family-uniform:65536"]
    R = ref_gpu.RefSolver()
    for spec in specs:
        d, e, exact = load(spec)
        n = len(d)
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
        if exact is not None:
            err = float(np.max(np.abs(w - exact)) / np.max(np.abs(exact)))
        else:
            err = sampled_error(d, e, w)
        print(json.dumps({
            "impl": "reference CUDA prototype", "input": spec, "n": n, "solves": solves,
            "ms_median": float(np.median(times)), "ms_min": float(np.min(times)),
            "workspace_bytes": ref_gpu.workspace_size(n), "max_err_over_normT": err,
        }), flush=True)
    R.close()


if __name__ == "__main__":
    main()
