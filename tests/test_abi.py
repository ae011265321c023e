"""CPU tests of the C ABI: the library loads, exports exactly what
include/amgt_b200.h declares, and its host-side logic behaves (no kernel
launches here)."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "amgt_b200.h")


def _declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"AMGT_API[^;(]*?\b(amgt_\w+)\s*\(", text, flags=re.S)))


def test_header_declares_entry_points():
    names = _declared()
    for want in ("amgt_csr_to_bsr", "amgt_spmv", "amgt_spgemm", "amgt_bsr_free", "amgt_CSRSpGemm",
                 "amgt_CSRMatrixMatvec"):
        assert want in names


def test_library_exports_every_declared_symbol():
    from amgt_b200 import _lib

    L = _lib.lib()
    for name in _declared():
        assert hasattr(L, name), name
    assert set(_declared()) == set(_lib.SIGNATURES), "ctypes table and header disagree"
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (amgt_\w+)", out))
    assert exported == set(_declared())


def test_library_is_built_for_sm100a_only():
    # the build passes exactly one -gencode, sm_100a; the device side of
    # this is test_gpu_hypre.py::test_kernels_run_sm100_code (binaryVersion)
    from amgt_b200 import build

    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_amg_setup_rejects_bad_params_without_a_device():
    from amgt_b200 import _lib

    L = _lib.lib()
    A = _lib.AmgtCsr(8, 8, 0, None, None, None)
    h = ctypes.c_void_p()
    for field, bad in (("max_iter", 0), ("max_iter", -3), ("tol", -1.0), ("tol", float("nan")),
                       ("max_coarse_rows", 0), ("solver", 2), ("restart", 0), ("restart", 33),
                       ("inner_prec0", 4), ("inner_tol", -1.0), ("max_outer", 0)):
        p = _lib.AmgtAmgParams()
        L.amgt_amg_default_params(ctypes.byref(p))
        p.solver = _lib.SOLVER_FGMRES_IR
        setattr(p, field, bad)
        assert L.amgt_amg_setup(ctypes.byref(A), 0, None, ctypes.byref(p), ctypes.byref(h), None) == 1, field
        assert not h.value


def test_kernel_arch_query_without_a_device():
    import torch

    from amgt_b200 import _lib

    v = ctypes.c_int(-1)
    rc = _lib.lib().amgt_kernel_arch(ctypes.byref(v))
    if not torch.cuda.is_available():
        assert rc == 6 and v.value == 0


def test_precision_policy_defaults_and_override():
    from amgt_b200 import _lib

    L = _lib.lib()
    # get_calculationPrecison: 0 -> double, 1 -> float, >= 2 -> half
    assert [L.amgt_precision_for_level(l) for l in range(5)] == [0, 1, 2, 2, 2]
    arr = (ctypes.c_int * 4)(0, 0, 1, 3)
    assert L.amgt_set_level_policy(arr, 4) == 0
    assert [L.amgt_precision_for_level(l) for l in range(7)] == [0, 0, 1, 3, 3, 3, 3]
    bad = (ctypes.c_int * 1)(9)
    assert L.amgt_set_level_policy(bad, 1) == 1
    assert L.amgt_set_level_policy(None, 0) == 0
    assert [L.amgt_precision_for_level(l) for l in range(3)] == [0, 1, 2]
    # the SpGEMM engine switch: AUTO / CUDA_CORE / TENSOR_CORE only
    assert L.amgt_spgemm_set_engine(3) == 1 and L.amgt_spgemm_set_engine(-1) == 1
    assert L.amgt_spgemm_set_engine(2) == 0 and L.amgt_spgemm_set_engine(0) == 0


def test_invalid_arguments_are_rejected_without_a_device():
    from amgt_b200 import _lib

    L = _lib.lib()
    assert L.amgt_spmv(0, 1.0, None, None, 0.0, None, None) == 1
    assert L.amgt_spgemm(0, None, None, None, None, None) == 1
    assert L.amgt_csr_to_bsr(None, None, None) == 1
    assert L.amgt_CSRMatrixMatvec(0, 1.0, None, None, 0.0, None, 0) == 1
    assert L.amgt_status_string(1) == b"invalid argument"
    assert L.amgt_set_allocator(ctypes.c_void_p(1), None, None) == 1


def test_mirror_matrix_create_destroy_host_only():
    from amgt_b200 import _lib

    L = _lib.lib()
    h = L.amgt_CSRMatrixCreate(8, 8, 0, None, None, None, 3)
    assert h
    assert h.contents.coasen_level == 3 and ord(h.contents.bsr_tag) == 0
    assert L.amgt_CSRMatrixDestroy(h) == 0
    assert not L.amgt_CSRMatrixCreate(-1, 8, 0, None, None, None, 0)
    # BoomerAMG entry points: argument checks before any device work
    A = _lib.AmgtBsr()
    A.row, A.col = 8, 4  # not square
    P = _lib.AmgtCsr()
    assert L.amgt_boomer_interp(ctypes.byref(A), None, ctypes.byref(P), None, None) == 1
    assert L.amgt_boomer_interp(None, None, ctypes.byref(P), None, None) == 1
    assert L.amgt_boomer_hierarchy_levels(None) == 0
    assert L.amgt_boomer_hierarchy_level(None, 0, None, None) == 1
    assert L.amgt_boomer_free_host(None) == 1


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES", None) == "", reason="explicitly hidden GPU")
def test_init_reports_device_state():
    import torch

    from amgt_b200 import _lib

    rc = _lib.lib().amgt_init()
    assert rc == (0 if torch.cuda.is_available() else 6)
