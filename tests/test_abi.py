"""C-ABI library: loads, exports every entry point of include/brdc.h, and
answers the argument checks that need no GPU."""
import ctypes
import os
import re

import pytest

import brdc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "brdc.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b(brdc_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_matches_binding_list():
    assert sorted(brdc.EXPORTS) == declared_symbols()


def test_library_exports_every_declared_symbol(built_lib):
    lib = ctypes.CDLL(built_lib)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_workspace_query(built_lib):
    assert brdc.workspace_size(1) > 0
    small, big = brdc.workspace_size(4096), brdc.workspace_size(65536)
    assert big > small
    # O(n): far below the reference's n*min(n,4096) delta slab
    assert big < 400 * 65536
    assert big % 256 == 0
    with pytest.raises(brdc.BrdcError) as ei:
        brdc.workspace_size(0)
    assert ei.value.status == brdc.INVALID_VALUE
    with pytest.raises(brdc.BrdcError):
        brdc.workspace_size(-5)


def test_argument_checks_without_device(built_lib):
    lib = brdc.load()
    # NULL handle first, as tridiag_solver.cu:2545-2547
    assert lib.brdc_dstebr(None, 10, None, None, None, None, 0) == brdc.INVALID_HANDLE
    assert lib.brdc_get_info(None, None, None) == brdc.INVALID_HANDLE
    assert lib.brdc_destroy(None) == brdc.INVALID_HANDLE
    assert lib.brdc_create(None) == brdc.INVALID_POINTER
    assert brdc.load().brdc_status_to_string(9) == b"not_converged"
    assert brdc.load().brdc_status_to_string(4) == b"invalid_workspace"


def test_lapack_style_query(built_lib):
    # cpu/src/dstedc_dc_br.f:44-75 query and argument errors
    info, lw, liw = brdc.dstedc_dc_br_query(4096)
    assert info == 0 and liw == 7 * 4096 and lw % 4096 == 0 and lw >= 18 * 4096
    assert brdc.dstedc_dc_br_query(20)[1:] == (1, 1)
    assert brdc.dstedc_dc_br_query(-1)[0] == -1
    assert brdc.dstedc_dc_br_query(4096, lwork=10, liwork=7 * 4096)[0] == -5
    assert brdc.dstedc_dc_br_query(4096, lwork=10**6, liwork=5)[0] == -7


def test_batched_workspace_query(built_lib):
    assert brdc.batched_workspace_size([0, 10, 50, 4146]) > brdc.workspace_size(4096)
    with pytest.raises(brdc.BrdcError):
        brdc.batched_workspace_size([0, 10, 10])


def test_noalloc_scratch_covers_its_limit(built_lib):
    # brdc_dstebr_noalloc solves n <= 16384 in a 6 MiB static device array
    # (brdc_capi.cu kNoAllocBytes); the workspace layout must stay within it.
    assert brdc.workspace_size(16384) <= 6 * 2**20


def _header_symbols(name, pattern):
    text = open(os.path.join(ROOT, "include", name)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(pattern + r"\s*\(", text)))


def test_lapack_names_exported(built_lib):
    names = _header_symbols("brdc_lapack.h", r"\b((?:dstebr_|sstebr_|LAPACKE_[a-z_]+))")
    assert names == ["LAPACKE_dstebr", "LAPACKE_dstebr_work", "LAPACKE_sstebr",
                     "LAPACKE_sstebr_work", "dstebr_", "sstebr_"]
    lib = ctypes.CDLL(built_lib)
    for name in names:
        assert hasattr(lib, name), name


def test_input_generators_exported(built_lib):
    import build as brdc_build

    lib = ctypes.CDLL(brdc_build.INPUTLIB)
    for name in _header_symbols("brdc_inputs.h", r"\b(brdc_[a-z0-9_]+)"):
        assert hasattr(lib, name), name


def _fortran_query(fn, ctype, n, lwork=-1, liwork=-1):
    ci = ctypes.c_int
    w = (ctype * 1)()
    iw = (ci * 1)()
    info = ci(7)
    d = (ctype * max(n, 1))()
    e = (ctype * max(n, 1))()
    fn(ctypes.byref(ci(n)), d, e, w, ctypes.byref(ci(lwork)), iw, ctypes.byref(ci(liwork)),
       ctypes.byref(info))
    return info.value, w[0], iw[0]


@pytest.mark.parametrize("name, ctype", [("dstebr_", ctypes.c_double), ("sstebr_", ctypes.c_float)])
def test_stebr_query_and_argument_errors(built_lib, name, ctype):
    # the DSTEDC_DC_BR query and errors (cpu/src/dstedc_dc_br.f:44-75) under
    # the upstream names; none of these touch the GPU
    fn = getattr(ctypes.CDLL(built_lib), name)
    info, lw, liw = _fortran_query(fn, ctype, 4096)
    ref = brdc.dstedc_dc_br_query(4096)
    assert info == 0 and (int(lw), liw) == ref[1:]
    assert _fortran_query(fn, ctype, 20)[1:] == (1.0, 1)
    assert _fortran_query(fn, ctype, -1)[0] == -1
    assert _fortran_query(fn, ctype, 4096, lwork=10, liwork=7 * 4096)[0] == -5
    assert _fortran_query(fn, ctype, 4096, lwork=10**6, liwork=5)[0] == -7
    # orders 0 and 1 need no solve
    assert _fortran_query(fn, ctype, 0, 1, 1)[0] == 0
    assert _fortran_query(fn, ctype, 1, 1, 1)[0] == 0


@pytest.mark.parametrize("name, ctype", [("LAPACKE_dstebr", ctypes.c_double),
                                         ("LAPACKE_sstebr", ctypes.c_float)])
def test_lapacke_checks_without_device(built_lib, name, ctype):
    fn = getattr(ctypes.CDLL(built_lib), name)
    fn.restype = ctypes.c_int
    d = (ctype * 4)(1.0, 2.0, float("nan"), 4.0)
    e = (ctype * 3)(0.5, 0.5, 0.5)
    assert fn(4, d, e) == -2
    d = (ctype * 4)(1.0, 2.0, 3.0, 4.0)
    e = (ctype * 3)(0.5, float("nan"), 0.5)
    assert fn(4, d, e) == -3
    assert fn(-2, d, e) == -1
    one = (ctype * 1)(3.25)
    assert fn(1, one, (ctype * 1)()) == 0 and one[0] == 3.25


def test_vectors_workspace_query(built_lib):
    lib = brdc.load()
    nb = ctypes.c_size_t(0)
    assert lib.brdc_dstebr_vectors_workspace_size(4096, ctypes.byref(nb)) == brdc.SUCCESS
    # the checkpoints plus M (n^2) and two half-size eigenvector buffers
    assert nb.value >= 16 * 4096 * 4096 and nb.value % 256 == 0
    assert lib.brdc_dstebr_vectors_workspace_size(0, ctypes.byref(nb)) == brdc.INVALID_VALUE
    assert lib.brdc_dstebr_vectors_workspace_size(1 << 20, ctypes.byref(nb)) == brdc.INVALID_VALUE
    assert lib.brdc_dstebr_vectors(None, 10, None, None, None, None, 10, None, 0) == brdc.INVALID_HANDLE
