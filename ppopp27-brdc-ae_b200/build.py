"""Build the sm_100a solver library in-tree.

``python build.py`` (or ``brdc.build.build()``) compiles
``csrc/brdc_capi.cu`` with nvcc into ``brdc/libbrdc_b200.so``, the host
copy of the secular state machine into ``brdc/libbrdc_hostcheck.so`` (used by
the CPU tests only) and the reference bench's input generators
(``csrc/brdc_inputs.cpp``) into ``brdc/libbrdc_inputs.so``.  nvcc
cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "brdc")
LIB = os.path.join(OUT, "libbrdc_b200.so")
HOSTLIB = os.path.join(OUT, "libbrdc_hostcheck.so")
INPUTLIB = os.path.join(OUT, "libbrdc_inputs.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    deps = _sources() + [os.path.join(HERE, "..", "include", h) for h in ("brdc.h", "brdc_lapack.h")] + [__file__]
    deps = [d for d in deps if not d.endswith(("host_check.cpp", "brdc_inputs.cpp"))]
    if force or _stale(LIB, deps):
        cmd = [_nvcc(), *NVCC_FLAGS, "-o", LIB, os.path.join(CSRC, "brdc_capi.cu")]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    hdeps = [os.path.join(CSRC, "host_check.cpp"), os.path.join(CSRC, "brdc_secular.cuh")]
    if force or _stale(HOSTLIB, hdeps):
        subprocess.run(
            [cxx, "-O2", "-fPIC", "-shared", "-std=c++17", "-o", HOSTLIB,
             os.path.join(CSRC, "host_check.cpp")],
            check=True,
        )
    ideps = [os.path.join(CSRC, "brdc_inputs.cpp"), os.path.join(HERE, "..", "include", "brdc_inputs.h")]
    if force or _stale(INPUTLIB, ideps):
        subprocess.run(
            [cxx, "-O2", "-fPIC", "-shared", "-std=c++17", "-o", INPUTLIB, ideps[0]],
            check=True,
        )
    return LIB


def nvcc_shared(src: str, out: str, deps=(), includes=(), force: bool = False) -> str:
    """Compile one stand-alone .cu file into a shared library for sm_100a
    (the bench's FP64 probe and test helpers use it), when out is stale."""
    if force or _stale(out, [src, *deps]):
        cmd = [_nvcc(), *NVCC_FLAGS, *[f"-I{d}" for d in includes], "-o", out, src]
        subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
