"""Input files and the reference's own input generators.

* ``.de.bin`` files (gpu/bench/tridiag_dc_bench.cu:393-447): an int64 order n,
  then either the compact payload -- n doubles of D, n-1 of E -- or a dense
  n x n column-major matrix whose diagonal and first subdiagonal are the
  tridiagonal.  :func:`read_de` accepts both, :func:`write_de` writes the
  compact form; any other payload size is an error, as in the reference.
* :func:`generate` -- the GPU bench's data modes ("bench", "test", and its
  "normal", "uniform", "toeplitz", "clustered"; tridiag_dc_bench.cu:229-339),
  computed in ``libbrdc_inputs.so`` with the same C++ <random> engines and
  seeds.
* :func:`spectrum_case` -- the spectrum-prescribed matrices of the paper's
  accuracy and timing figures (cpu/jobs/run_spectrum_de_cache_job.sh:52-110):
  LAPACK DLATMS builds a symmetric tridiagonal (KL = KU = 1, PACK = 'B') with a
  random spectrum -- MODE 6 with DIST 'U' or 'N' -- or a clustered one --
  MODE 1, COND 1e12: one eigenvalue of modulus 1, the other n-1 of modulus
  1e-12 -- seeded ISEED = (1, 2, n mod 4093 + MODE, 5).  The fourth case is the
  Toeplitz matrix D = 2, E = 1/4.  DLATMS comes from the LAPACK in scipy's
  bundled OpenBLAS; its bulge chase costs O(n^2) (about 9 s at n = 16,384, 140 s
  at 65,536 on one host core), which is why the reference caches the results
  as ``.de.bin`` files: :func:`write_spectrum_cache` writes the same cache.

``python -m brdc.inputs spectrum-cache OUTDIR [--sizes 8192,16384]`` writes
the cache and prints the reference job's manifest lines;
``python -m brdc.inputs generate MODE N OUT.de.bin [--index I]`` writes one
generated matrix.
"""
from __future__ import annotations

import ctypes
import glob
import os
import sys
from typing import Iterable, List, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
INPUT_LIB_PATH = os.path.join(_HERE, "libbrdc_inputs.so")

GPU_BENCH_MODES = ("bench", "test", "normal", "uniform", "toeplitz", "clustered")
SPECTRUM_MODES = ("uniform", "normal", "toeplitz", "clustered")
SPECTRUM_SIZES = (8192, 16384, 32768, 49152, 65536)
# (DIST, MODE, COND) of each DLATMS case (run_spectrum_de_cache_job.sh:80-86)
_DLATMS_CASES = {
    "uniform": (b"U", 6, 1.0),
    "normal": (b"N", 6, 1.0),
    "clustered": (b"U", 1, 1.0e12),
}


# --------------------------------------------------------------------------
# .de.bin files
# --------------------------------------------------------------------------

def read_de(path: str) -> Tuple[np.ndarray, np.ndarray]:
    """(D[n], E[n-1]) of a ``.de.bin`` file, compact or dense payload
    (read_tridiagonal_file, tridiag_dc_bench.cu:393-433)."""
    total = os.path.getsize(path)
    with open(path, "rb") as f:
        head = f.read(8)
        if len(head) != 8:
            raise ValueError(f"invalid tridiagonal header in file: {path}")
        n = int(np.frombuffer(head, dtype="<i8")[0])
        if n <= 0:
            raise ValueError(f"invalid tridiagonal header in file: {path}")
        payload = total - 8
        if payload == (2 * n - 1) * 8:
            d = np.fromfile(f, dtype="<f8", count=n)
            e = np.fromfile(f, dtype="<f8", count=n - 1)
            if d.size != n or e.size != n - 1:
                raise ValueError(f"failed to read compact tridiagonal payload: {path}")
            return d.astype(np.float64), e.astype(np.float64)
        if payload == n * n * 8:
            m = np.fromfile(f, dtype="<f8", count=n * n)
            if m.size != n * n:
                raise ValueError(f"failed to read dense tridiagonal payload: {path}")
            # column-major: entry (row, col) sits at row + col*n, so the
            # row-major view indexes [col, row]
            m = m.reshape(n, n)
            return np.diagonal(m).astype(np.float64), np.diagonal(m, offset=1).astype(np.float64)
    raise ValueError(f"unsupported tridiagonal file payload bytes={payload} for n={n} in {path}")


def write_de(path: str, d, e) -> None:
    """Write the compact ``.de.bin`` form (write_tridiagonal_file,
    tridiag_dc_bench.cu:435-447)."""
    d = np.ascontiguousarray(d, dtype="<f8")
    e = np.ascontiguousarray(e, dtype="<f8")
    n = d.size
    if n < 1 or e.size != n - 1:
        raise ValueError(f"need D[n] and E[n-1] with n >= 1 (got {d.size}, {e.size})")
    with open(path, "wb") as f:
        f.write(np.asarray([n], dtype="<i8").tobytes())
        f.write(d.tobytes())
        f.write(e.tobytes())


# --------------------------------------------------------------------------
# The GPU bench's generators
# --------------------------------------------------------------------------

_ilib = None


def _input_lib():
    global _ilib
    if _ilib is None:
        if not os.path.exists(INPUT_LIB_PATH):
            raise RuntimeError(f"{INPUT_LIB_PATH} is missing: build it with build.py")
        lib = ctypes.CDLL(INPUT_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        lib.brdc_input_generate.argtypes = [ctypes.c_char_p, ctypes.c_int64, ctypes.c_int64, dp, dp]
        lib.brdc_input_generate.restype = ctypes.c_int
        _ilib = lib
    return _ilib


def generate(mode: str, n: int, index: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    """(D[n], E[n-1]) of one of the GPU bench's data modes; ``index`` is the
    position of n in the bench's size list (it seeds the "bench" mode)."""
    if mode not in GPU_BENCH_MODES:
        raise ValueError(f"unsupported data mode {mode!r}: expected one of {GPU_BENCH_MODES}")
    n = int(n)
    if n < 1:
        raise ValueError("n must be >= 1")
    d = np.empty(n, dtype=np.float64)
    e = np.empty(max(n - 1, 1), dtype=np.float64)
    dp = ctypes.POINTER(ctypes.c_double)
    rc = _input_lib().brdc_input_generate(
        mode.encode(), n, int(index), d.ctypes.data_as(dp), e.ctypes.data_as(dp)
    )
    if rc != 0:
        raise ValueError(f"brdc_input_generate({mode!r}, {n}) failed ({rc})")
    return d, e[: n - 1].copy()


# --------------------------------------------------------------------------
# Spectrum-prescribed matrices (LAPACK DLATMS)
# --------------------------------------------------------------------------

_lapack = None


def _lapack_lib():
    global _lapack
    if _lapack is None:
        import scipy

        libs = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
        cands = sorted(glob.glob(os.path.join(libs, "libscipy_openblas*.so*")))
        if not cands:
            raise RuntimeError("scipy's OpenBLAS (LAPACK DLATMS) not found under " + libs)
        _lapack = ctypes.CDLL(cands[0])
    return _lapack


def dlatms_tridiagonal(n: int, dist: bytes, mode: int, cond: float, iseed):
    """LAPACK DLATMS(n, n, dist, iseed, 'S', eig, mode, cond, 1, 1, 1, 'B', ...):
    a symmetric tridiagonal with the spectrum that MODE/COND prescribe.
    Returns (prescribed eigenvalues, D, E, info)."""
    n = int(n)
    ci, cd = ctypes.c_int, ctypes.c_double
    seed = (ci * 4)(*[int(s) for s in iseed])
    eig = np.zeros(n)
    ab = np.zeros((n, 2))  # Fortran AB(2, n): row 1 the diagonal, row 2 the subdiagonal
    work = np.zeros(3 * n)
    info = ci(0)
    vp = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    one = ctypes.c_size_t(1)
    _lapack_lib().scipy_dlatms_(
        ctypes.byref(ci(n)), ctypes.byref(ci(n)), ctypes.c_char_p(dist), seed,
        ctypes.c_char_p(b"S"), vp(eig), ctypes.byref(ci(int(mode))), ctypes.byref(cd(float(cond))),
        ctypes.byref(cd(1.0)), ctypes.byref(ci(1)), ctypes.byref(ci(1)), ctypes.c_char_p(b"B"),
        vp(ab), ctypes.byref(ci(2)), vp(work), ctypes.byref(info), one, one, one,
    )
    return eig, ab[:, 0].copy(), ab[: n - 1, 1].copy(), int(info.value)


def spectrum_case(mode: str, n: int):
    """(D, E, info, prescribed eigenvalues or None) of one case of the paper's
    spectrum cache (fill_case, run_spectrum_de_cache_job.sh:66-87)."""
    n = int(n)
    if mode == "toeplitz":
        return np.full(n, 2.0), np.full(max(n - 1, 0), 0.25), 0, None
    if mode not in _DLATMS_CASES:
        raise ValueError(f"unsupported spectrum mode {mode!r}: expected one of {SPECTRUM_MODES}")
    dist, md, cond = _DLATMS_CASES[mode]
    eig, d, e, info = dlatms_tridiagonal(n, dist, md, cond, (1, 2, n % 4093 + md, 5))
    return d, e, info, eig


def write_spectrum_cache(outdir: str, sizes: Iterable[int] = SPECTRUM_SIZES,
                         modes: Iterable[str] = SPECTRUM_MODES, out=sys.stdout) -> List[str]:
    """Write ``{mode}_{n}.de.bin`` for every mode and size, as the reference's
    cache job does, and print its manifest (mode,n,path,generator,info)."""
    os.makedirs(outdir, exist_ok=True)
    lines = ["mode,n,path,generator,info"]
    for mode in modes:
        for n in sizes:
            d, e, info, _ = spectrum_case(mode, n)
            path = os.path.join(outdir, f"{mode}_{int(n)}.de.bin")
            if info == 0:
                write_de(path, d, e)
            gen = "structured_toeplitz" if mode == "toeplitz" else "dlatms_symmetric_band"
            lines.append(f"{mode},{int(n)},{path},{gen},{info}")
    if out is not None:
        for ln in lines:
            print(ln, file=out)
    return lines


def _main(argv) -> int:
    import argparse

    ap = argparse.ArgumentParser(prog="python -m brdc.inputs")
    sub = ap.add_subparsers(dest="cmd", required=True)
    sc = sub.add_parser("spectrum-cache", help="write the spectrum-prescribed .de.bin cache")
    sc.add_argument("outdir")
    sc.add_argument("--sizes", default=",".join(str(s) for s in SPECTRUM_SIZES))
    sc.add_argument("--modes", default=",".join(SPECTRUM_MODES))
    g = sub.add_parser("generate", help="write one GPU-bench data mode as .de.bin")
    g.add_argument("mode", choices=GPU_BENCH_MODES)
    g.add_argument("n", type=int)
    g.add_argument("out")
    g.add_argument("--index", type=int, default=0)
    a = ap.parse_args(argv)
    if a.cmd == "spectrum-cache":
        lines = write_spectrum_cache(
            a.outdir, [int(s) for s in a.sizes.split(",") if s], [m for m in a.modes.split(",") if m]
        )
        with open(os.path.join(a.outdir, "manifest.csv"), "w") as f:
            f.write("\n".join(lines) + "\n")
    else:
        d, e = generate(a.mode, a.n, a.index)
        write_de(a.out, d, e)
    return 0


if __name__ == "__main__":
    sys.exit(_main(sys.argv[1:]))
