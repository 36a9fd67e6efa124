"""Benchmark of the B200 BR values-only tridiagonal eigensolver.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline workload: one plain values-only solve of order N = 65,536, FP64,
uniform family (D, E iid U(0,1), seeded), the configuration whose GPU time
the reference publishes (60.5 ms on H100-PCIe).  A step is one solve with D
and E already resident in HBM; L2 is flushed (256 MiB write) before every
timed solve, outside the timed interval, and each solve is timed with CUDA
events on its stream.  value = mean ms per solve (lower is better).

Also reported on the same line: the e2e time through the C ABI's
host-buffer entry brdc_dstebr_host with pinned buffers (H2D of D and E,
solve, D2H of W inside the timed interval),
the per-phase roofline of the dominant kernel (FP64 pipe or HBM), the other
three families at the same order, accuracy against the oracle, workspace
bytes, clocks sampled during the timed loop, and the CPU baseline: the
oracle (C restatement of the reference's DSTEDC_DC_BR, OpenMP on all host
threads) timed on a bounded sample of the same workload.

--input PATH.de.bin or --data MODE[:N] replace the headline input with a
file in the reference's .de.bin format or one of the reference's own
generators (its GPU bench's data modes, or the paper's DLATMS
spectrum-prescribed matrices as spectrum-MODE); the default line also carries
those inputs at N = 8,192 under "paper_inputs".

--impl reference times the reference's CPU implementation of this path
(the oracle port; no Fortran compiler exists in the image) on the same
workload and prints the same metric with "impl": "reference".

With --gpus N > 1 (torchrun, one process per GPU) every rank solves its own
replica (a single solve does not shard: the tree funnels into one root
merge); value is the max over ranks of the per-solve time and
solves_per_s is the whole-job rate.  The batch of config 3 does shard:
"sharded_batch" gives its whole-job solves/s with each rank solving its
share of the 4096 instances (no collective on the data path).

Beside this build, the default line times the reference CUDA prototype
(built from the reference's sources into oracle/_ref) on the same inputs on
the same GPU ("ref_gpu"), and records whether cuSOLVER exports
cusolverDnXstedc.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ppopp27-brdc-ae_b200"))

METRIC = "ms/solve N=65,536 FP64 (fwd; fwd+bwd) and batched solves/s, vs plain & CPU"
N_HEAD = 65536
FAMILY_HEAD = "uniform"


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        try:
            with open(path) as f:
                p = json.load(f)
            return float(p["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def start_clock_sampler(path):
    try:
        return subprocess.Popen(
            ["nvidia-smi",
             "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
             "--format=csv,noheader,nounits", "-lms", "50"],
            stdout=open(path, "w"), stderr=subprocess.DEVNULL)
    except Exception:
        return None


def stop_clock_sampler(proc, path, device_index):
    if proc is None:
        return None
    proc.terminate()
    try:
        proc.wait(timeout=5)
    except Exception:
        proc.kill()
    sm, smax, reasons = [], 0.0, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    try:
        for line in open(path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9 or parts[0] != str(device_index):
                continue
            sm.append(float(parts[1]))
            smax = max(smax, float(parts[2]))
            for nm, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "1", "yes"):
                    reasons.add(nm)
    except Exception:
        return None
    if not sm:
        return None
    return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
            "samples": len(sm)}


class quiet_host:
    """The events of a timed loop made beforehand, and Python's garbage
    collector paused while it runs: every timed interval opens with an
    event and then waits for the host to submit the work, so a collection
    pass or an allocation on the host would be timed as solve time."""

    def __init__(self, torch, steps):
        self.ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(steps)]

    def __enter__(self):
        import gc

        self.was = gc.isenabled()
        gc.disable()
        return self.ev

    def __exit__(self, *exc):
        import gc

        if self.was:
            gc.enable()
        return False


def time_solves(torch, solver, D, E, W, ws, steps, flush):
    """Per-solve device times (ms) with an L2 flush before each solve."""
    stream = torch.cuda.current_stream()
    times = []
    with quiet_host(torch, steps) as ev:
        for e0, e1 in ev:
            flush.zero_()
            e0.record(stream)
            solver.dstebr(D, E, W=W, workspace=ws)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    return times


def cpu_reference_times(d, e, budget_s, min_solves=1, max_solves=50):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    oracle.set_threads(os.cpu_count() or 1)
    threads = oracle.max_threads()
    oracle.dstedc_dc_br(d, e)  # warm-up
    times = []
    t_end = time.perf_counter() + budget_s
    while len(times) < max_solves and (len(times) < min_solves or time.perf_counter() < t_end):
        t0 = time.perf_counter()
        oracle.dstedc_dc_br(d, e)
        times.append((time.perf_counter() - t0) * 1e3)
    return times, threads


def run_reference_arm(args, rank):
    if rank != 0:
        return
    d, e, name, data, _ = load_workload(args.input, args.data)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    oracle.set_threads(os.cpu_count() or 1)
    threads = oracle.max_threads()
    for _ in range(args.warmup):
        oracle.dstedc_dc_br(d, e)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.dstedc_dc_br(d, e)
        times.append((time.perf_counter() - t0) * 1e3)
    v = float(np.mean(times))
    line = {
        "impl": "reference",
        "metric": f"ms/solve FP64, {name}" if (args.input or args.data) else METRIC,
        "value": v,
        "unit": "ms",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": v,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": data,
        "config": {"workload": name, "n": len(d)},
        "cpu_baseline": {"value": v, "unit": "ms", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full solves of the workload"},
        "e2e": {"value": v, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference CPU path DSTEDC_DC_BR restated in C (oracle/brdc_oracle.c); "
                "no Fortran compiler in the image",
    }
    print(json.dumps(line), flush=True)


def run_profile_case(spec):
    """One or more plain solves of a seeded instance with the library's
    default launch shapes, nothing else on the GPU: solve i launches k_init,
    k_norm, k_subtree, then per level above the subtree k_level and k_sweeps
    (from the second solve on as a replay of the library's graph of the
    same launches), so a kernel's launch index is known in advance."""
    import torch

    import brdc
    from brdc import families

    parts = spec.split(":")
    if parts[0] == "vectors":
        # vectors:family:n -- one eigenvector solve (brdc_dstebr_vectors)
        fam, n = parts[1], int(parts[2])
        d, e = families.generate(fam, n)
        solver = brdc.Solver()
        W, Z = solver.dstebr_vectors(torch.tensor(d, device="cuda"), torch.tensor(e, device="cuda"))
        torch.cuda.synchronize()
        solver.close()
        return
    fam, n = parts[0], int(parts[1])
    solves = int(parts[2]) if len(parts) > 2 else 1
    adjoint = len(parts) > 3 and parts[3] == "bwd"
    d, e = families.generate(fam, n)
    solver = brdc.Solver()
    D = torch.tensor(d, device="cuda")
    E = torch.tensor(e, device="cuda")
    W = torch.empty(n, dtype=torch.float64, device="cuda")
    ws = solver.checkpoint_workspace(n) if adjoint else solver.workspace(n)
    G = torch.ones(n, dtype=torch.float64, device="cuda")
    for _ in range(solves):
        solver.dstebr(D, E, W=W, workspace=ws)
        if adjoint:
            solver.dstebr_backward(D, E, G, workspace=ws, keep_forward=True)
    torch.cuda.synchronize()
    solver.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--profile-case", default=None,
                    help="family:n[:solves[:bwd]] -- run that many plain solves (default 1) of "
                         "the seeded instance, each followed by the adjoint with bwd, and exit; "
                         "vectors:family:n -- one eigenvector solve; a fixed launch sequence "
                         "for profilers")
    ap.add_argument("--input", default=None,
                    help="solve the tridiagonal of a .de.bin file instead of the headline input")
    ap.add_argument("--data", default=None,
                    help="MODE[:N] -- solve one of the reference's inputs instead: bench, test, "
                         "normal, uniform, toeplitz, clustered (its GPU bench's generators), "
                         "spectrum-{uniform,normal,clustered,toeplitz} (the paper's DLATMS cache) "
                         "or family-{uniform,normal,toeplitz,clustered} (the plain-solve families)")
    args = ap.parse_args()
    if args.profile_case:
        run_profile_case(args.profile_case)
        return
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    if args.input or args.data:
        if rank == 0:
            run_input_workload(args)
        return

    import torch

    import brdc
    from brdc import families

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist = dist_mod
        # rank 0 alone measures the extras (minutes) while the others wait
        # at the closing barrier
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))

    solver = brdc.Solver()
    d, e = families.generate(FAMILY_HEAD, N_HEAD, instance=rank)
    D = torch.tensor(d, device="cuda")
    E = torch.tensor(e, device="cuda")
    W = torch.empty(N_HEAD, dtype=torch.float64, device="cuda")
    ws = solver.workspace(N_HEAD)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")

    # the library's autotuner picks the launch shapes for this input
    # (outside the timed region); the line reports its choice
    tuning = solver.autotune(D, E, workspace=ws)
    for _ in range(args.warmup):
        solver.dstebr(D, E, W=W, workspace=ws)
    torch.cuda.synchronize()
    info = solver.info(N_HEAD, ws)

    clocks_path = os.path.join("/tmp", f"brdc_clocks_{os.getpid()}.csv")
    sampler = start_clock_sampler(clocks_path) if rank == 0 else None
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    times = time_solves(torch, solver, D, E, W, ws, args.steps, flush)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = stop_clock_sampler(sampler, clocks_path, local_rank) if rank == 0 else None
    from brdc.sharding import max_over_ranks

    ms = max_over_ranks(float(np.mean(times)), dist, device="cuda")
    # kernels the last timed solve ran, and whether the library replayed
    # them from its graph (every solve after the first two with these buffers)
    launch_rec = solver.last_launches()

    # config 3's batch sharded over the ranks (every rank takes part)
    sharded = None
    if world > 1 and not args.no_extras:
        sharded = bench_sharded_batch(torch, brdc, families, rank, world, dist, flush)

    extras = {}
    if rank == 0 and not args.no_extras:
        extras = collect_extras(torch, brdc, families, solver, D, E, W, ws, d, e, flush, args,
                                head_ms=ms)

    if rank == 0:
        diag = solver.diagnostics(N_HEAD, ws)
        line = {
            "metric": METRIC,
            "value": ms,
            "unit": "ms",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms,
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded uniform U(0,1) family, numpy PCG64 [1, N, rank])",
            "config": {
                "workload": f"plain values-only BR solve, {FAMILY_HEAD} family, N={N_HEAD}",
                "n": N_HEAD, "family": FAMILY_HEAD,
                "l2": "flushed by a 256 MiB write before every timed solve (outside the timed interval)",
                "parallelism": f"replicas x{world}",
                "tuning": tuning,
            },
            "solves_per_s": world * 1000.0 / ms,
            "info": info,
            "gpu_launches": launch_rec["launches"],
            "launch_path": "graph replay" if launch_rec["replayed"] else "stream launches",
            "ms_min": float(np.min(times)),
            "ms_median": float(np.median(times)),
            "workspace_bytes": ws.numel(),
            "deflation_K_per_level": [lv["dd_after_sum"] for lv in diag["level"]],
            "secular_iters_per_level": [
                [round(lv["secular_iter_sum"] / max(lv["dd_after_sum"], 1), 2), lv["secular_iter_max"],
                 lv["secular_iter_failed"], lv["threads_per_root"]] for lv in diag["level"]],
            "clocks": clocks,
        }
        line.update({k: v for k, v in extras.items() if k != "launches"})
        if sharded is not None:
            line["sharded_batch"] = sharded
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def dsterf(d, e):
    """LAPACK DSTERF eigenvalues (scipy's bundled LAPACK), ascending."""
    import scipy.linalg.lapack as la

    w, info = la.dsterf(np.array(d, dtype=np.float64), np.array(e, dtype=np.float64))
    if info != 0:
        raise RuntimeError(f"dsterf info {info}")
    return np.sort(w)


def lapack_sample_error(d, e, w, blocks=16, width=4):
    """Max |w_i - lambda_i| / ||T|| over a sample of eigenvalues computed by
    LAPACK bisection (DSTEBZ through scipy): `blocks` evenly spread runs of
    `width` consecutive indices, the first and last included, so the check
    costs O(n * blocks * width) instead of DSTERF's O(n^2)."""
    import scipy.linalg

    n = len(d)
    starts = np.unique(np.linspace(0, max(n - width, 0), blocks).astype(int))
    worst = 0.0
    ext = scipy.linalg.eigvalsh_tridiagonal(d, e, select="i", select_range=(0, 0),
                                            lapack_driver="stebz")
    ext2 = scipy.linalg.eigvalsh_tridiagonal(d, e, select="i", select_range=(n - 1, n - 1),
                                             lapack_driver="stebz")
    norm = max(abs(ext[0]), abs(ext2[0]))
    for st in starts:
        hi = min(st + width - 1, n - 1)
        ref = scipy.linalg.eigvalsh_tridiagonal(d, e, select="i", select_range=(int(st), int(hi)),
                                                lapack_driver="stebz")
        worst = max(worst, float(np.max(np.abs(w[st:hi + 1] - ref))))
    return worst / norm


def bench_config2(torch, families, solver, flush):
    """The plain-solve table over orders and families: median ms of 10
    solves after 3 warm-ups (default launch shapes), eigenvalues/s, max
    error over ||T|| (Toeplitz: every eigenvalue against its closed form;
    the others: 64 sampled eigenvalues against LAPACK bisection), workspace
    bytes and the non-deflated pole count per level."""
    table = []
    for n in (8192, 16384, 32768, 49152, 65536):
        ws = solver.workspace(n)
        W = torch.empty(n, dtype=torch.float64, device="cuda")
        for fam in ("uniform", "normal", "toeplitz", "clustered"):
            d, e = families.generate(fam, n)
            Dt = torch.tensor(d, device="cuda")
            Et = torch.tensor(e, device="cuda")
            for _ in range(3):
                solver.dstebr(Dt, Et, W=W, workspace=ws)
            torch.cuda.synchronize()
            tt = time_solves(torch, solver, Dt, Et, W, ws, 10, flush)
            ms = float(np.median(tt))
            w = W.cpu().numpy()
            if fam == "toeplitz":
                ref = families.toeplitz_eigenvalues(n)
                err = float(np.max(np.abs(w - ref)) / np.max(np.abs(ref)))
            else:
                err = lapack_sample_error(d, e, w)
            dg = solver.diagnostics(n, ws)
            table.append({"n": n, "family": fam, "ms": ms, "eigenvalues_per_s": n * 1e3 / ms,
                          "max_err_over_normT": err, "workspace_bytes": ws.numel(),
                          "K_per_level": [lv["dd_after_sum"] for lv in dg["level"]]})
        solver._ws.clear()
    return table


def measure_e2e(torch, solver, D, E, W, ws, d, e, flush, warmup, steps):
    """The solve end to end through the C ABI's host-buffer entry
    (brdc_dstebr_host): pinned host D and E copied in, the solve, W copied
    back, all inside the timed interval.  D, E and W are the device-entry
    arguments of the headline line: their solve is the reference for the
    host entry's result, and the same end-to-end interval is also timed
    through the device entry with the copies made by the caller."""
    n = len(d)
    solver.dstebr(D, E, W=W, workspace=ws)
    ref = W.cpu().numpy()
    # one pinned buffer [D | E]: the entry copies it in one piece
    hDE = torch.cat([torch.tensor(d), torch.tensor(e, dtype=torch.float64)]).pin_memory()
    hD, hE = hDE[:n], hDE[n:]
    hW = torch.empty(n, dtype=torch.float64).pin_memory()
    hws = solver.host_workspace(n)
    stream = torch.cuda.current_stream()
    # the C entry called as a C caller would, with its arguments prepared
    # once, so that no Python-side argument handling sits in the interval
    # before the first copy is enqueued
    import ctypes

    import brdc

    call = brdc.load().brdc_dstebr_host
    argv = (solver.h, n, ctypes.c_void_p(hD.data_ptr()), ctypes.c_void_p(hE.data_ptr()),
            ctypes.c_void_p(hW.data_ptr()), ctypes.c_void_p(hws.data_ptr()), hws.numel())
    e2e = []
    with quiet_host(torch, warmup + steps) as ev:
        for i, (e0, e1) in enumerate(ev):
            flush.zero_()
            e0.record(stream)
            st = call(*argv)
            e1.record(stream)
            e1.synchronize()
            if st != 0:
                raise RuntimeError(f"brdc_dstebr_host returned {st}")
            if i >= warmup:
                e2e.append(e0.elapsed_time(e1))
    err = float(np.max(np.abs(hW.numpy() - ref)))
    # the same through the device entry, the copies made by the caller
    DE = torch.empty(n + len(e), dtype=torch.float64, device=D.device)
    Dv, Ev = DE[:n], DE[n:]
    dev = []
    with quiet_host(torch, warmup + steps) as ev:
        for i, (e0, e1) in enumerate(ev):
            flush.zero_()
            e0.record(stream)
            DE.copy_(hDE, non_blocking=True)
            solver.dstebr(Dv, Ev, W=W, workspace=ws)
            hW.copy_(W, non_blocking=True)
            e1.record(stream)
            e1.synchronize()
            if i >= warmup:
                dev.append(e0.elapsed_time(e1))
    return {"value": float(np.mean(e2e)), "unit": "ms",
            "h2d_bytes_per_step": int((hD.numel() + hE.numel()) * 8),
            "d2h_bytes_per_step": int(hW.numel() * 8),
            "entry": ("brdc_dstebr_host on pinned host buffers: k_norm reads D and E and the "
                      "top level writes W through their mapped addresses, over PCIe inside "
                      "the timed interval"),
            "max_abs_diff_vs_device_entry": err,
            "device_entry_with_caller_copies_ms": float(np.mean(dev))}


def load_workload(input_path, data_spec):
    """(d, e, workload name, data description, exact spectrum or None).

    --input PATH reads a .de.bin file (compact or dense payload);
    --data MODE[:N] generates one of the reference's inputs: the GPU bench's
    modes (bench, test, normal, uniform, toeplitz, clustered) or the paper's
    spectrum-prescribed cache (spectrum-uniform, spectrum-normal,
    spectrum-clustered through LAPACK DLATMS, spectrum-toeplitz) or the
    plain-solve families (family-uniform, family-normal, family-toeplitz,
    family-clustered); N defaults to 65,536.  Without either, the headline
    uniform family."""
    from brdc import families, inputs

    if input_path:
        d, e = inputs.read_de(input_path)
        return d, e, f"file {os.path.basename(input_path)}, N={len(d)}", "file (.de.bin)", None
    if data_spec:
        mode, _, n = data_spec.partition(":")
        n = int(n) if n else N_HEAD
        if mode.startswith("spectrum-"):
            m = mode[len("spectrum-"):]
            d, e, info, eig = inputs.spectrum_case(m, n)
            if info != 0:
                raise RuntimeError(f"DLATMS info {info} for {mode}:{n}")
            exact = np.sort(eig) if eig is not None else families.toeplitz_eigenvalues(n, 2.0, 0.25)
            return (d, e, f"spectrum-prescribed {m} (paper cache), N={n}",
                    "LAPACK DLATMS spectrum-prescribed tridiagonal" if eig is not None
                    else "Toeplitz D=2, E=1/4", exact)
        if mode.startswith("family-"):
            fam = mode[len("family-"):]
            d, e = families.generate(fam, n)
            exact = families.toeplitz_eigenvalues(n) if fam == "toeplitz" else None
            return (d, e, f"plain values-only BR solve, {fam} family, N={n}",
                    f"synthetic (seeded {fam} family)", exact)
        d, e = inputs.generate(mode, n)
        exact = families.toeplitz_eigenvalues(n, 2.0, 0.25) if mode == "toeplitz" else None
        return d, e, f"reference GPU-bench data mode {mode}, N={n}", f"reference generator ({mode})", exact
    d, e = families.generate(FAMILY_HEAD, N_HEAD)
    return (d, e, f"plain values-only BR solve, {FAMILY_HEAD} family, N={N_HEAD}",
            "synthetic (seeded uniform U(0,1) family)", None)


def input_error(d, e, w, exact):
    """max |w - lambda| / ||T||: against the exact spectrum where the input
    prescribes one, else against LAPACK bisection on sampled eigenvalues."""
    if exact is not None:
        return float(np.max(np.abs(w - exact)) / max(np.max(np.abs(exact)), 1e-300))
    return lapack_sample_error(d, e, w)


def run_input_workload(args):
    """One plain solve per step of the workload --input or --data names, on
    one GPU; the line carries the same timing keys as the headline's."""
    import torch

    import brdc

    d, e, name, data, exact = load_workload(args.input, args.data)
    n = len(d)
    solver = brdc.Solver()
    D = torch.tensor(d, device="cuda")
    E = torch.tensor(e if len(e) else np.zeros(1), device="cuda")
    W = torch.empty(n, dtype=torch.float64, device="cuda")
    ws = solver.workspace(n)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    tuning = solver.autotune(D, E, workspace=ws)
    for _ in range(args.warmup):
        solver.dstebr(D, E, W=W, workspace=ws)
    torch.cuda.synchronize()
    clocks_path = os.path.join("/tmp", f"brdc_clocks_{os.getpid()}.csv")
    sampler = start_clock_sampler(clocks_path)
    times = time_solves(torch, solver, D, E, W, ws, args.steps, flush)
    torch.cuda.synchronize()
    clocks = stop_clock_sampler(sampler, clocks_path, torch.cuda.current_device())
    ms = float(np.mean(times))
    launches = solver.last_launches()["launches"]
    err = input_error(d, e, W.cpu().numpy(), exact)
    line = {
        "metric": f"ms/solve FP64, {name}", "value": ms, "unit": "ms", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": data,
        "config": {"workload": name, "n": n, "tuning": tuning,
                   "l2": "flushed by a 256 MiB write before every timed solve (outside the timed interval)"},
        "info": solver.info(n, ws), "max_err_over_normT": err,
        "e2e": measure_e2e(torch, solver, D, E, W, ws, d, e, flush, args.warmup, args.steps),
        "gpu_launches": launches, "ms_median": float(np.median(times)), "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    solver.close()


def bench_paper_inputs(torch, solver, flush, n=8192):
    """The reference's own inputs at one order: its GPU bench's data modes
    and the paper's spectrum-prescribed matrices (DLATMS), each solved with
    the default launch shapes -- median ms of 5 solves and the max error over
    ||T|| (against the prescribed spectrum where there is one)."""
    from brdc import inputs

    out = {"n": n}
    ws = solver.workspace(n)
    W = torch.empty(n, dtype=torch.float64, device="cuda")
    specs = [m for m in inputs.GPU_BENCH_MODES] + ["spectrum-" + m for m in ("uniform", "normal", "clustered")]
    for spec in specs:
        d, e, _, _, exact = load_workload(None, f"{spec}:{n}")
        Dt = torch.tensor(d, device="cuda")
        Et = torch.tensor(e, device="cuda")
        for _ in range(3):
            solver.dstebr(Dt, Et, W=W, workspace=ws)
        torch.cuda.synchronize()
        tt = time_solves(torch, solver, Dt, Et, W, ws, 5, flush)
        out[spec] = {"ms": float(np.median(tt)),
                     "max_err_over_normT": input_error(d, e, W.cpu().numpy(), exact)}
    solver._ws.clear()
    return out


def bench_vectors(torch, brdc, families, sizes=(4096, 16384)):
    """The eigenvector path (brdc_dstebr_vectors) on the normal family:
    median ms of 3 calls, max |Z^T Z - I| and max |T Z - Z diag(W)| / ||T||
    (computed on the device)."""
    import ctypes

    out = {}
    solver = brdc.Solver()
    for n in sizes:
        d, e = families.generate("normal", n)
        D = torch.tensor(d, device="cuda")
        E = torch.tensor(e, device="cuda")
        nb = ctypes.c_size_t(0)
        brdc.load().brdc_dstebr_vectors_workspace_size(n, ctypes.byref(nb))
        ws = torch.empty(nb.value, dtype=torch.uint8, device="cuda")
        W, Z = solver.dstebr_vectors(D, E, workspace=ws)
        ts = []
        for _ in range(3):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            W, Z = solver.dstebr_vectors(D, E, workspace=ws)
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        Zc = Z.contiguous()
        orth = (Zc.t() @ Zc - torch.eye(n, dtype=torch.float64, device="cuda")).abs().max().item()
        TZ = D[:, None] * Zc
        TZ[:-1] += E[:, None] * Zc[1:]
        TZ[1:] += E[:, None] * Zc[:-1]
        res = (TZ - Zc * W[None, :]).abs().max().item() / W.abs().max().item()
        ms = float(np.median(ts))
        out[str(n)] = {"ms": ms, "max_orth_err": orth, "max_residual_over_normT": res,
                       "workspace_bytes": nb.value}
        del ws, Z, Zc, TZ
        torch.cuda.empty_cache()
    solver.close()
    return out


def xstedc_probe():
    """Whether cuSOLVER on this machine exports cusolverDnXstedc, the
    routine the reference's GPU bench compares against
    (gpu/bench/tridiag_dc_bench.cu:1144, 1277): an exported-name lookup of
    each libcusolver the process can find, nothing more."""
    import ctypes
    import glob

    cands = sorted(set(glob.glob("/usr/local/cuda/lib64/libcusolver.so*")))
    try:
        import nvidia.cusolver as nc

        cands += sorted(glob.glob(os.path.join(list(nc.__path__)[0], "lib", "libcusolver.so*")))
    except Exception:
        pass
    found = []
    for path in cands:
        try:
            lib = ctypes.CDLL(path)
        except OSError:
            continue
        found.append({"library": path, "exports_cusolverDnXstedc": hasattr(lib, "cusolverDnXstedc")})
    exported = any(f["exports_cusolverDnXstedc"] for f in found)
    return {"libraries": found, "available": exported,
            "note": None if exported else "unavailable on this box: no cuSOLVER here exports "
                                          "cusolverDnXstedc"}


def ref_gpu_times(torch, R, D, E, W, steps, warmup, flush):
    """Per-solve device times (ms) of the reference CUDA prototype on its own
    stream, with the same L2 flush before every timed solve as ours."""
    with torch.cuda.stream(R.stream):
        for _ in range(warmup):
            R.solve(D, E, W)
        R.stream.synchronize()
        times = []
        for _ in range(steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(R.stream)
            R.solve(D, E, W)
            e1.record(R.stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    return times


def bench_ref_gpu(torch, families, solver, flush, args, head_ms, fam_ms, paper):
    """The reference CUDA prototype (the reference's gpu/src, compiled for
    sm_100a from its own sources into oracle/_ref and called through its
    solve entry tridiag_solver_run_from_device_tridiagonal,
    gpu/src/tridiag_solver.cu:2541) timed on this GPU in this run, beside
    this build, on the same inputs with the same L2 flush: the four families
    at the headline order (the headline family with the headline's warm-up
    and at most 50 timed solves), the reference GPU bench's own data modes at the headline order
    (this build timed beside it with its default launch shapes), and the
    paper inputs at 8,192 whose times this line already carries.  A
    comparison leg only: nothing of it is this build's timed work."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_gpu
    from brdc import inputs

    out = {"cusolver_xstedc": xstedc_probe()}
    if not ref_gpu.available():
        out["unavailable"] = "oracle/_ref not built: the reference tree was absent when building"
        return out
    R = ref_gpu.RefSolver()
    try:
        rows = {}
        Wr = torch.empty(N_HEAD, dtype=torch.float64, device="cuda")

        def row(spec, d, e, exact, steps, warmup, ours_ms):
            Dt = torch.tensor(d, device="cuda")
            Et = torch.tensor(e, device="cuda")
            W1 = torch.empty(len(d), dtype=torch.float64, device="cuda") if len(d) != N_HEAD else Wr
            tt = ref_gpu_times(torch, R, Dt, Et, W1, steps, warmup, flush)
            ms = float(np.mean(tt))
            err = input_error(d, e, np.sort(W1.cpu().numpy()), exact)
            rows[spec] = {"ms": ms, "ms_median": float(np.median(tt)), "solves": steps,
                          "workspace_bytes": ref_gpu.workspace_size(len(d)),
                          "max_err_over_normT": err, "ours_ms": ours_ms,
                          "speedup": ms / ours_ms if ours_ms else None}

        for fam in ("uniform", "normal", "toeplitz", "clustered"):
            d, e = families.generate(fam, N_HEAD)
            exact = families.toeplitz_eigenvalues(N_HEAD) if fam == "toeplitz" else None
            head = fam == FAMILY_HEAD
            row(f"family-{fam}:{N_HEAD}", d, e, exact,
                min(args.steps, 50) if head else (3 if fam == "toeplitz" else 5),
                args.warmup if head else 1, head_ms if head else fam_ms.get(fam))
        # the reference GPU bench's data modes at the headline order; this
        # build with its default launch shapes on the same inputs
        saved = solver.tuning()
        solver.set_tuning(**DEFAULT_TUNING)
        ws = solver.workspace(N_HEAD)
        for mode in inputs.GPU_BENCH_MODES:
            if mode == "test":
                continue  # the bench's small self-test mode
            d, e, _, _, exact = load_workload(None, f"{mode}:{N_HEAD}")
            Dt = torch.tensor(d, device="cuda")
            Et = torch.tensor(e, device="cuda")
            for _ in range(2):
                solver.dstebr(Dt, Et, W=Wr, workspace=ws)
            torch.cuda.synchronize()
            ours = float(np.mean(time_solves(torch, solver, Dt, Et, Wr, ws, 5, flush)))
            row(f"{mode}:{N_HEAD}", d, e, exact, 3, 1, ours)
        solver.set_tuning(**saved)
        # the paper inputs at the order bench_paper_inputs used
        n = paper["n"]
        for spec, rec in paper.items():
            if spec == "n":
                continue
            d, e, _, _, exact = load_workload(None, f"{spec}:{n}")
            row(f"{spec}:{n}", d, e, exact, 3, 1, rec["ms"])
        out.update(rows[f"family-{FAMILY_HEAD}:{N_HEAD}"])
        out["rows"] = rows
    finally:
        R.close()
        solver._ws.clear()
    return out


def collect_extras(torch, brdc, families, solver, D, E, W, ws, d, e, flush, args, head_ms=None):
    out = {}
    headline_tuning = solver.tuning()

    # accuracy of the headline solve against LAPACK bisection (DSTEBZ) on
    # 128 sampled eigenvalues, extremes included
    solver.dstebr(D, E, W=W, workspace=ws)
    w = W.cpu().numpy()
    out["max_err_vs_lapack_sample"] = lapack_sample_error(d, e, w, blocks=32, width=4)

    # per-phase timings and roofline of the dominant kernel
    solver.set_timing(True)
    keys = ("leaf_ms", "merge_ms", "secular_ms", "lowner_ms", "rows_ms", "total_ms")
    acc = {k: 0.0 for k in keys}
    level_acc = None
    reps = 5
    launches = 0
    for _ in range(reps):
        flush.zero_()
        solver.dstebr(D, E, W=W, workspace=ws)
        t = solver.last_timings()
        for k in keys:
            acc[k] += t[k] / reps
        launches = t["launches"]
        if level_acc is None:
            level_acc = [[0.0] * 4 for _ in t["level_ms"]]
        for k2, row in enumerate(t["level_ms"]):
            for j in range(4):
                level_acc[k2][j] += row[j] / reps
    acc["level_ms"] = level_acc
    solver.set_timing(False)
    out["launches"] = launches
    out["phase_ms"] = acc
    diag = solver.diagnostics(N_HEAD, ws)
    fused = t["fused_levels"]
    out["roofline"] = roofline(diag, acc, N_HEAD, fused=fused,
                               level_rows=headline_tuning["fused_level_rows"])

    # other families at the same order
    fam_ms = {}
    fam_tuning = {}
    for fam in ("normal", "toeplitz", "clustered"):
        dd, ee = families.generate(fam, N_HEAD)
        Df = torch.tensor(dd, device="cuda")
        Ef = torch.tensor(ee, device="cuda")
        fam_tuning[fam] = solver.autotune(Df, Ef, workspace=ws)
        # two untimed solves: the second captures the graph the timed ones replay
        for _ in range(2):
            solver.dstebr(Df, Ef, W=W, workspace=ws)
        torch.cuda.synchronize()
        tt = time_solves(torch, solver, Df, Ef, W, ws, 3, flush)
        fam_ms[fam] = float(np.mean(tt))
        if fam == "toeplitz":
            err = np.max(np.abs(W.cpu().numpy() - families.toeplitz_eigenvalues(N_HEAD))) / 4.0
            out["toeplitz_max_err_vs_closed_form"] = float(err)
            dg = solver.diagnostics(N_HEAD, ws)
            out["toeplitz_roofline"] = roofline(dg, None, N_HEAD, total_ms=fam_ms[fam],
                                                fused=fused, level_rows=0)
    out["family_ms"] = fam_ms
    out["family_tuning"] = fam_tuning
    solver.set_tuning(**headline_tuning)

    out["e2e"] = measure_e2e(torch, solver, D, E, W, ws, d, e, flush, args.warmup, args.steps)

    solver.set_tuning(**DEFAULT_TUNING)
    out["config2"] = bench_config2(torch, families, solver, flush)
    out["paper_inputs"] = bench_paper_inputs(torch, solver, flush)
    out["vectors"] = bench_vectors(torch, brdc, families)
    solver.set_tuning(**headline_tuning)
    out["fwd_bwd"] = bench_fwd_bwd(torch, families, solver, flush, args)
    out["batched"] = bench_batched(torch, brdc, families, solver, flush)
    out["fit"] = bench_fit(torch, brdc, families, flush)
    out["ref_gpu"] = bench_ref_gpu(torch, families, solver, flush, args, head_ms, fam_ms,
                                   out["paper_inputs"])

    # CPU baseline: the oracle on a bounded sample of the same workload
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    cpu_t, threads = cpu_reference_times(d, e, args.cpu_budget)
    # LAPACK DSTERF (scipy's bundled LAPACK, one host thread) beside it, on
    # a bounded sample: the n = 16384 instance of the same family (DSTERF is
    # O(n^2); the full order would take most of a minute)
    ds, es = families.generate(FAMILY_HEAD, 16384)
    t0 = time.perf_counter()
    dsterf(ds, es)
    out["dsterf_cpu"] = {"value": (time.perf_counter() - t0) * 1e3, "unit": "ms", "cores": 1,
                         "sample": "one solve of the uniform n = 16384 instance"}
    out["cpu_baseline"] = {"value": float(np.median(cpu_t)), "unit": "ms", "cores": threads,
                           "kind": "port",
                           "sample": f"{len(cpu_t)} full solves of the headline input "
                                     f"(oracle restatement of DSTEDC_DC_BR, OpenMP)"}
    return out


def _event_ms(torch, fn, reps, flush, stream=None):
    stream = stream or torch.cuda.current_stream()
    out = []
    with quiet_host(torch, reps) as ev:
        for e0, e1 in ev:
            flush.zero_()
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            out.append(e0.elapsed_time(e1))
    return float(np.mean(out))


def bench_fwd_bwd(torch, families, solver, flush, args):
    """Differentiated solve, normal family, L = sum g_i lambda_i: forward
    with checkpoints plus the adjoint, against the plain forward."""
    res = {}
    for n in (4096, 16384, N_HEAD):
        d, e = families.generate("normal", n)
        D = torch.tensor(d, device="cuda")
        E = torch.tensor(e, device="cuda")
        G = torch.tensor(np.random.Generator(np.random.PCG64([2, n, 1])).standard_normal(n),
                         device="cuda")
        W = torch.empty(n, dtype=torch.float64, device="cuda")
        gD = torch.empty(n, dtype=torch.float64, device="cuda")
        gE = torch.empty(n, dtype=torch.float64, device="cuda")
        ws = solver.workspace(n)
        wsc = solver.checkpoint_workspace(n)

        def fwd():
            solver.dstebr(D, E, W=W, workspace=ws)

        def fwd_c():
            solver.dstebr(D, E, W=W, workspace=wsc)

        def bwd():
            solver.dstebr_backward(D, E, G, workspace=wsc, keep_forward=True, gD=gD, gE=gE)

        def both():
            fwd_c()
            bwd()

        reps = 20

        def timed(fn):
            # each pattern warmed right before its timing, so that the
            # library captures its graphs (forward, adjoint) outside it
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            return _event_ms(torch, fn, reps, flush)

        t_f = timed(fwd)
        t_fc = timed(fwd_c)
        t_fb = timed(both)
        res[str(n)] = {"fwd_ms": t_f, "fwd_checkpointed_ms": t_fc, "fwd_bwd_ms": t_fb,
                       "bwd_ms": t_fb - t_fc, "ratio_fwd_bwd_to_fwd": t_fb / t_f,
                       "workspace_bytes": ws.numel(), "checkpoint_workspace_bytes": wsc.numel()}
        del ws, wsc
        solver._ws.clear()
    return {"family": "normal", "loss": "sum g_i lambda_i, g ~ N(0,1)",
            "l2": "flushed before every timed call", "by_n": res}


def bench_batched(torch, brdc, families, solver, flush):
    """4096 tridiagonals, N log-uniform in [32, 8192], the four families
    mixed: one batched solve replayed from a CUDA graph, against looping the
    plain single-matrix entry over the same instances."""
    count = 4096
    off, D, E, orders, fams = families.batch(count, 32, 8192, seed=3)
    Dt = torch.tensor(D, device="cuda")
    Et = torch.tensor(E, device="cuda")
    W = torch.empty(int(off[-1]), dtype=torch.float64, device="cuda")
    ws = solver.batched_workspace(off)
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        solver.set_stream(stream)
        tuning = solver.autotune(Dt, Et, offsets=off, workspace=ws)
        solver.dstebr_batched(off, Dt, Et, W=W, workspace=ws)  # uploads the forest tables
        stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            solver.dstebr_batched(off, Dt, Et, W=W, workspace=ws)
        g.replay()
        stream.synchronize()
        t_graph = _event_ms(torch, g.replay, 5, flush, stream)
        t_eager = _event_ms(torch, lambda: solver.dstebr_batched(off, Dt, Et, W=W, workspace=ws),
                            5, flush, stream)
    solver.set_stream(torch.cuda.current_stream())
    torch.cuda.synchronize()
    Wb = W.cpu().numpy()
    del g

    # the plain entry looped over the instances, one shared workspace, with
    # the library's default launch shapes
    solver.set_tuning(**DEFAULT_TUNING)
    nmax = int(np.max(orders))
    ws1 = solver.workspace(nmax)
    W1 = torch.empty_like(W)
    views = [(Dt[int(off[b]):int(off[b + 1])], Et[int(off[b]):int(off[b + 1]) - 1],
              W1[int(off[b]):int(off[b + 1])]) for b in range(count)]

    def loop():
        for Db, Eb, Wb_ in views:
            solver.dstebr(Db, Eb if Eb.numel() else Db, W=Wb_, workspace=ws1)

    loop()
    torch.cuda.synchronize()
    t_loop = _event_ms(torch, loop, 1, flush)
    same = float(np.max(np.abs(W1.cpu().numpy() - Wb)))

    # per-instance error against LAPACK on every 16th instance
    import scipy.linalg

    errs = []
    for b in range(0, count, 16):
        lo, hi = int(off[b]), int(off[b + 1])
        ref = scipy.linalg.eigvalsh_tridiagonal(D[lo:hi], E[lo:hi - 1])
        errs.append(float(np.max(np.abs(Wb[lo:hi] - ref)) / np.max(np.abs(ref))))
    return {"count": count, "orders": "log-uniform [32, 8192]", "rows": int(off[-1]),
            "tuning": tuning,
            "families": "uniform, normal, toeplitz, clustered in turn",
            "graph_ms": t_graph, "eager_batched_ms": t_eager, "looped_plain_ms": t_loop,
            "solves_per_s": count * 1e3 / t_graph,
            "looped_solves_per_s": count * 1e3 / t_loop,
            "speedup_vs_looped": t_loop / t_graph,
            "max_abs_diff_batched_vs_looped": same,
            "max_rel_err_vs_lapack": max(errs),
            "lapack_sample": f"{len(errs)} instances (every 16th)",
            "workspace_bytes": ws.numel()}


def bench_sharded_batch(torch, brdc, families, rank, world, dist, flush):
    """Config 3's batch (4096 tridiagonals, N log-uniform in [32, 8192], the
    four families in turn) sharded over the ranks: each rank solves its
    partition_instances share (balanced by sum n^2) as one batched solve
    replayed from a CUDA graph, with no collective on the data path.  Time =
    max over ranks of the mean of 5 replays (L2 flushed before each);
    solves_per_s is the whole job's rate."""
    from brdc.sharding import max_over_ranks, pack, partition_instances

    count = 4096
    off, D, E, orders, _ = families.batch(count, 32, 8192, seed=3)
    idx = partition_instances(orders, world)[rank]
    o2, D2, E2 = pack(off, D, E, idx)
    solver = brdc.Solver()
    Dt = torch.tensor(D2, device="cuda")
    Et = torch.tensor(E2, device="cuda")
    W = torch.empty(int(o2[-1]), dtype=torch.float64, device="cuda")
    ws = solver.batched_workspace(o2)
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        solver.set_stream(stream)
        solver.set_tuning(subtree_levels=5)
        solver.dstebr_batched(o2, Dt, Et, W=W, workspace=ws)  # writes the forest tables
        stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            solver.dstebr_batched(o2, Dt, Et, W=W, workspace=ws)
        g.replay()
        stream.synchronize()
        t = float(np.mean(_event_ms(torch, g.replay, 5, flush, stream)))
    torch.cuda.synchronize()
    info = solver.info_status(0, ws)[0]
    del g
    solver.close()
    t_max = max_over_ranks(t, dist, device="cuda")
    sum_n2 = float(np.sum(np.asarray(orders, dtype=np.float64)[idx] ** 2))
    sum_n2_max = max_over_ranks(sum_n2, dist, device="cuda")
    return {"count": count, "ranks": world, "ms": t_max, "solves_per_s": count * 1e3 / t_max,
            "balance_sum_n2_max_over_mean": sum_n2_max / (float(np.sum(orders.astype(np.float64) ** 2)) / world),
            "info_rank0": info,
            "timing": "max over ranks of each rank's mean graph replay (5, L2 flushed before each)"}


def bench_fit(torch, brdc, families, flush, steps=200, lr=0.1):
    """Inverse eigenvalue fit: 1024 tridiagonals, N log-uniform in [64,
    4096], normal family; loss sum (lambda_i - t_i)^2 with targets the
    eigenvalues of a second seeded tridiagonal of the same N; 200 gradient
    steps (batched forward with checkpoints, batched adjoint, update of D
    and E) captured in one CUDA graph."""
    count = 1024
    orders = families.batch_orders(count, 64, 4096, seed=4)
    off = np.zeros(count + 1, dtype=np.int64)
    off[1:] = np.cumsum(orders)
    tot = int(off[-1])
    D = np.empty(tot)
    E = np.zeros(tot)
    D2 = np.empty(tot)
    E2 = np.zeros(tot)
    for b, n in enumerate(orders):
        d, e = families.generate("normal", int(n), instance=1 + b)
        d2, e2 = families.generate("normal", int(n), instance=100001 + b)
        D[off[b]:off[b + 1]] = d
        E[off[b]:off[b + 1] - 1] = e
        D2[off[b]:off[b + 1]] = d2
        E2[off[b]:off[b + 1] - 1] = e2
    s = brdc.Solver()
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        s.set_stream(stream)
        T = s.dstebr_batched(off, torch.tensor(D2, device="cuda"), torch.tensor(E2, device="cuda"))
        Dt = torch.tensor(D, device="cuda")
        Et = torch.tensor(E, device="cuda")
        D0, E0 = Dt.clone(), Et.clone()
        W = torch.empty(tot, dtype=torch.float64, device="cuda")
        G = torch.empty_like(W)
        gD = torch.empty_like(W)
        gE = torch.empty_like(W)
        hist = torch.zeros(steps + 1, dtype=torch.float64, device="cuda")
        ws = s.batched_workspace(off, checkpoints=True)
        tuning = s.autotune(Dt, Et, offsets=off, workspace=ws)
        Dt.copy_(D0)

        def step(i):
            s.dstebr_batched(off, Dt, Et, W=W, workspace=ws)
            torch.sub(W, T, out=G)
            hist[i].copy_(torch.dot(G, G))
            G.mul_(2.0)
            s.dstebr_batched_backward(off, Dt, Et, G, workspace=ws, keep_forward=True, gD=gD, gE=gE)
            Dt.add_(gD, alpha=-lr)
            Et.add_(gE, alpha=-lr)

        step(0)  # uploads the forest tables
        stream.synchronize()
        t_eager = _event_ms(torch, lambda: step(0), 3, flush, stream)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            for i in range(steps):
                step(i)
        Dt.copy_(D0)
        Et.copy_(E0)
        stream.synchronize()
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.replay()
        e1.record(stream)
        e1.synchronize()
        t_graph = e0.elapsed_time(e1)
        s.dstebr_batched(off, Dt, Et, W=W, workspace=ws)
        torch.sub(W, T, out=G)
        hist[steps].copy_(torch.dot(G, G))
        stream.synchronize()
        h = hist.cpu().numpy()
    del g
    s.close()
    return {"count": count, "orders": "log-uniform [64, 4096]", "rows": tot, "steps": steps,
            "tuning": tuning,
            "lr": lr, "graph_ms_total": t_graph, "ms_per_step_graph": t_graph / steps,
            "ms_per_step_eager": t_eager, "steps_per_s": steps * 1e3 / t_graph,
            "optimizer": "SGD", "loss_first": float(h[0]), "loss_last": float(h[steps]),
            "loss_at": {str(k): float(h[k]) for k in (1, 10, 50, 100, 199)},
            "checkpoint_workspace_bytes": ws.numel()}


def work_model(diag, fused):
    """Algorithmic FP64 work of the solve from the solver's own counters
    (a divide or square root counts as one flop, an FMA as two):
      leaf Jacobi     (12 s + 15) flops per rotation, s(s-1)/2 rotations a
                      sweep, summed over the leaves with the sweeps each
                      leaf's half-warp ran
      secular         8 flops per pole-root pair and sweep; sweeps per root
                      = its iterations + the initial midpoint sweep
      Loewner         4 flops per pair (inner merges only)
      boundary rows   10 flops per pair (inner merges only)
    Returns (flops of the subtree kernel, per-level dict for the rest)."""
    levels = diag["level"]
    nlev = len(levels)
    leaves = diag["leaf_count"]
    s = 16
    sweeps = diag.get("leaf_sweeps_sum") or leaves * diag["leaf_sweeps_max"]
    leaf = sweeps * (s * (s - 1) / 2) * (12 * s + 15)
    per = []
    for k, lv in enumerate(levels):
        kk = max(lv["dd_after_sum"], 1)
        sweeps = lv["secular_iter_sum"] / kk + 1.0
        sec = 8.0 * lv["dd_after_sq_sum"] * sweeps
        inner = k < nlev - 1
        low = 4.0 * lv["dd_after_sq_sum"] if inner else 0.0
        rows = 10.0 * lv["dd_after_sq_sum"] if inner else 0.0
        per.append((sec, low, rows))
    sub = leaf + sum(a + b + c for a, b, c in per[:fused])
    return sub, per


def roofline(diag, phase, n, total_ms=None, fused=0, level_rows=0):
    """Roofline of the dominant kernel (by measured time) against the
    measured FP64 FMA peak (flop model in work_model), or, for the
    per-level deflation, against HBM copy bandwidth (68 bytes per row and
    level: d, z, two rows read and written, an index).  Candidates: the
    subtree kernel (leaves and the lowest levels), k_level (the levels whose
    largest merge has at most `level_rows` rows: its phase column holds the
    whole level), k_sweeps (roots, Loewner, rows and placement of the other
    levels, and of the merges k_level hands on), and the per-level merge and
    deflation."""
    hbm, hbm_kind = measured_peaks()
    levels = diag["level"]
    fp64_peak = fp64_peak_gflops()
    sub_flops, per = work_model(diag, fused)
    res = {"pairs_sum_k2": int(sum(lv["dd_after_sq_sum"] for lv in levels))}
    if phase is None:
        flops = sub_flops + sum(a + b + c for a, b, c in per[fused:])
        ach = flops / (total_ms * 1e-3) / 1e12
        res.update({"bound": "fp64", "kernel": "whole solve", "achieved": ach,
                    "peak": fp64_peak / 1e3, "unit": "TFLOP/s", "frac": ach / (fp64_peak / 1e3),
                    "traffic": None, "peak_kind": "measured (DFMA probe)"})
        return res
    lvl_ms = [0.0, 0.0]       # k_level, per-level merge + deflation
    lvl_work = [0.0, 0.0]
    sw_ms, sw_work = 0.0, 0.0
    for k in range(fused, len(levels)):
        lv = levels[k]
        mmax = lv["size_sum"] // max(lv["merge_count"], 1)
        row = phase["level_ms"][k]
        flops = sum(per[k])
        if mmax <= level_rows:
            lvl_ms[0] += row[0]
            lvl_work[0] += flops
        else:
            lvl_ms[1] += row[0]
            lvl_work[1] += 68.0 * n
            sw_work += flops
        sw_ms += row[1] + row[2] + row[3]
    cand = {
        "k_subtree": (phase["leaf_ms"], sub_flops, "fp64"),
        "k_level": (lvl_ms[0], lvl_work[0], "fp64"),
        "k_sweeps": (sw_ms, sw_work, "fp64"),
        "k_merge+k_merge_deflate": (lvl_ms[1], lvl_work[1], "hbm"),
    }
    name = max(cand, key=lambda k: cand[k][0])
    ms, work, bound = cand[name]
    if bound == "fp64":
        ach = work / (ms * 1e-3) / 1e12
        res.update({"bound": "fp64", "kernel": name, "achieved": ach, "peak": fp64_peak / 1e3,
                    "unit": "TFLOP/s", "frac": ach / (fp64_peak / 1e3),
                    "traffic": KERNEL_TRAFFIC.get(name),
                    "peak_kind": "measured (DFMA probe)", "work_per_launch": work,
                    "kernel_ms": ms})
    else:
        ach = work / (ms * 1e-3) / 1e9
        res.update({"bound": "hbm", "kernel": name, "achieved": ach, "peak": hbm,
                    "unit": "GB/s", "frac": ach / hbm, "traffic": KERNEL_TRAFFIC.get(name),
                    "peak_kind": hbm_kind + " copy bandwidth", "work_per_launch": work,
                    "kernel_ms": ms})
    tot = max(sum(c[0] for c in cand.values()), 1e-9)
    res["phase_share"] = {k: v[0] / tot for k, v in cand.items()}
    return res


# DRAM bytes (read + write) of one launch, from the ncu captures summarised
# in profiles/ (uniform N=65536): the working set is L2-resident, so DRAM
# sees little more than the first touch of the inputs.
KERNEL_TRAFFIC = {"k_subtree": 1240320}

# the library's default launch shapes (brdc_tuning defaults)
DEFAULT_TUNING = {"subtree_levels": -1, "deflate_cluster": 16, "sweep_lanes_target": 303104,
                  "fused_level_rows": 1 << 30}


_FP64 = None


def fp64_probe_lib() -> str:
    """libbench_fp64.so beside this file (built from bench_fp64.cu when stale)."""
    import build as brdc_build

    return brdc_build.nvcc_shared(os.path.join(ROOT, "bench_fp64.cu"),
                                  os.path.join(ROOT, "libbench_fp64.so"))


def fp64_peak_gflops():
    global _FP64
    if _FP64 is None:
        import ctypes

        lib = ctypes.CDLL(fp64_probe_lib())
        lib.brdc_probe_dfma_gflops.restype = ctypes.c_double
        lib.brdc_probe_dfma_gflops.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        best = 0.0
        for _ in range(3):
            best = max(best, lib.brdc_probe_dfma_gflops(148 * 8, 256, 20000))
        _FP64 = best
    return _FP64


if __name__ == "__main__":
    main()
