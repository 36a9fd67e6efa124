"""Seeded synthetic tridiagonal families.

The reference defines its inputs only through generators
(gpu/bench/tridiag_dc_bench.cu:229-339, cpu/bench/bench_cpu_strong_scaling.f90:
85-154).  The families used here are the four of the plain-solve
configuration -- uniform U(0,1), normal N(0,1), Toeplitz (D=2, E=1, closed
form 2-2cos(k*pi/(N+1))) and clustered (8 centres in U(-1,1) plus 1e-10
noise, E = 1e-6*U(0,1)) -- drawn from numpy PCG64 seeded with
[family id, N, instance] (family ids 1..4), D first, then E.
"""
from __future__ import annotations

import numpy as np

FAMILY_ID = {"uniform": 1, "normal": 2, "toeplitz": 3, "clustered": 4}
FAMILIES = tuple(FAMILY_ID)


def generate(family: str, n: int, instance: int = 0):
    """(D[n], E[n-1]) of one seeded instance."""
    rng = np.random.Generator(np.random.PCG64([FAMILY_ID[family], int(n), int(instance)]))
    m = max(int(n) - 1, 0)
    if family == "uniform":
        d = rng.uniform(0.0, 1.0, n)
        e = rng.uniform(0.0, 1.0, m)
    elif family == "normal":
        d = rng.standard_normal(n)
        e = rng.standard_normal(m)
    elif family == "toeplitz":
        d = np.full(n, 2.0)
        e = np.ones(m)
    elif family == "clustered":
        centres = rng.uniform(-1.0, 1.0, 8)
        d = centres[rng.integers(0, 8, n)] + 1.0e-10 * rng.standard_normal(n)
        e = 1.0e-6 * rng.uniform(0.0, 1.0, m)
    else:
        raise ValueError(family)
    return d, e


def toeplitz_eigenvalues(n: int, a: float = 2.0, b: float = 1.0) -> np.ndarray:
    """Closed-form spectrum of the Toeplitz tridiagonal (a on the diagonal,
    b off it), ascending."""
    k = np.arange(1, n + 1)
    return np.sort(a - 2.0 * b * np.cos(k * np.pi / (n + 1)))


def batch_orders(count: int, lo: int, hi: int, seed: int = 0) -> np.ndarray:
    """Orders log-uniform in [lo, hi] (rounded), as in the batched configs."""
    rng = np.random.Generator(np.random.PCG64([99, int(count), int(seed)]))
    return np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), count))).astype(np.int64)


def batch(count: int, lo: int, hi: int, families=FAMILIES, seed: int = 0):
    """Packed batch: returns (offsets[count+1], D, E, orders, family names);
    instance i uses family families[i % len(families)] and its E slot at the
    last row is 0."""
    orders = batch_orders(count, lo, hi, seed)
    off = np.zeros(count + 1, dtype=np.int64)
    off[1:] = np.cumsum(orders)
    D = np.empty(int(off[-1]))
    E = np.zeros(int(off[-1]))
    fams = []
    for i, n in enumerate(orders):
        f = families[i % len(families)]
        d, e = generate(f, int(n), instance=i + 1 + 1000 * seed)
        D[off[i]:off[i + 1]] = d
        E[off[i]:off[i + 1] - 1] = e
        fams.append(f)
    return off, D, E, orders, fams
