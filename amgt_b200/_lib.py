"""ctypes binding of libamgt_b200.so (the C ABI in include/amgt_b200.h).

Loading fails loudly when the library is missing: there is no CPU or
pure-PyTorch fallback for any entry point.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libamgt_b200.so")

AMGT_OK = 0
STATUS = {0: "AMGT_OK", 1: "AMGT_ERR_INVALID", 2: "AMGT_ERR_ALLOC", 3: "AMGT_ERR_CUDA", 4: "AMGT_ERR_DEVICE",
          5: "AMGT_ERR_UNSUPPORTED", 6: "AMGT_ERR_NO_DEVICE", 7: "AMGT_ERR_TOO_LARGE"}
NOALLOC_MAX_SEGMENTS = 1 << 18  # AMGT_NOALLOC_MAX_SEGMENTS
DOUBLE, FLOAT, HALF, BF16 = 0, 1, 2, 3
SOLVER_PCG, SOLVER_FGMRES_IR = 0, 1

c_int, c_double, c_void_p = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
P = ctypes.POINTER


class AmgtCsr(ctypes.Structure):
    _fields_ = [("num_rows", c_int), ("num_cols", c_int), ("num_nonzeros", c_int),
                ("i", c_void_p), ("j", c_void_p), ("data", c_void_p)]


class AmgtBsr(ctypes.Structure):
    _fields_ = [("row", c_int), ("col", c_int), ("nnz", c_int), ("blc_row", c_int), ("blc_col", c_int),
                ("blc_num", c_int), ("stand", c_double), ("avg_nnz", c_double),
                ("blcPtr", c_void_p), ("blcIdx", c_void_p), ("blcVal", c_void_p), ("blcMap", c_void_p),
                ("warpnum", c_int), ("rowPtrbyWarp", c_void_p), ("rowIdxbyWarp", c_void_p),
                ("blcVal_fp32", c_void_p), ("blcVal_fp16", c_void_p), ("blcVal_bf16", c_void_p),
                ("max_blc_per_row", c_int), ("csr_nnz", c_int), ("exact_prec", c_int)]


class AmgtVector(ctypes.Structure):
    _fields_ = [("data", c_void_p), ("size", c_int), ("num_vectors", c_int), ("vecstride", c_int)]


class AmgtCSRMatrix(ctypes.Structure):
    _fields_ = [("coasen_level", c_int), ("bsr_spmv_balanced_tag", ctypes.c_char), ("bsr_tag", ctypes.c_char),
                ("mixed_precision_flag", ctypes.c_char), ("owns_data", ctypes.c_char),
                ("bsr_mat", P(AmgtBsr)), ("bsr_mat_T", P(AmgtBsr)), ("csr", AmgtCsr)]


class AmgtAmgParams(ctypes.Structure):
    _fields_ = [("max_levels", c_int), ("max_coarse_rows", c_int), ("tol", c_double), ("max_iter", c_int),
                ("relax_weight", c_double), ("flexible", c_int), ("use_graph", c_int),
                ("galerkin_by_level", c_int), ("smooth_prec0", c_int), ("packed", c_int),
                ("exact_storage", c_int), ("solver", c_int), ("restart", c_int), ("inner_tol", c_double),
                ("inner_prec0", c_int), ("max_outer", c_int)]


class AmgtPbsr(ctypes.Structure):
    _fields_ = [("row", c_int), ("col", c_int), ("blc_row", c_int), ("blc_col", c_int), ("blc_num", c_int),
                ("nnz", c_int), ("prec", c_int), ("blcPtr", c_void_p), ("blcIdx", c_void_p), ("blcMap", c_void_p),
                ("rowVoff", c_void_p), ("val", c_void_p), ("max_blc_per_row", c_int), ("blcVoff", c_void_p)]


class AmgtTuneResult(ctypes.Structure):
    _fields_ = [("count", c_int), ("candidate", c_int * 8), ("ms", ctypes.c_float * 8), ("choice", c_int)]


ENGINE_AUTO, ENGINE_CUDA_CORE, ENGINE_TENSOR_CORE = 0, 1, 2


class AmgtBoomerParams(ctypes.Structure):
    _fields_ = [("theta", c_double), ("max_row_sum", c_double), ("p_max", c_int), ("coarsen_type", c_int)]

# name -> (restype, argtypes); every symbol include/amgt_b200.h declares
SIGNATURES = {
    "amgt_status_string": (ctypes.c_char_p, [c_int]),
    "amgt_init": (c_int, []),
    "amgt_kernel_launch_count": (ctypes.c_uint64, []),
    "amgt_kernel_arch": (c_int, [P(c_int)]),
    "amgt_set_allocator": (c_int, [c_void_p, c_void_p, c_void_p]),
    "amgt_trim_pool": (c_int, [ctypes.c_size_t]),
    "amgt_precision_for_level": (c_int, [c_int]),
    "amgt_set_level_policy": (c_int, [P(c_int), c_int]),
    "amgt_csr_to_bsr": (c_int, [P(AmgtCsr), P(AmgtBsr), c_void_p]),
    "amgt_bsr_to_csr": (c_int, [P(AmgtBsr), P(AmgtCsr), c_void_p]),
    "amgt_bsr_balance": (c_int, [P(AmgtBsr), c_void_p]),
    "amgt_bsr_make_shadow": (c_int, [P(AmgtBsr), c_int, c_void_p]),
    "amgt_bsr_transpose": (c_int, [P(AmgtBsr), P(AmgtBsr), c_void_p]),
    "amgt_bsr_make_exact": (c_int, [P(AmgtBsr), c_void_p]),
    "amgt_bsr_free": (c_int, [P(AmgtBsr), c_void_p]),
    "amgt_csr_free": (c_int, [P(AmgtCsr), c_void_p]),
    "amgt_spmv": (c_int, [c_int, c_double, P(AmgtBsr), c_void_p, c_double, c_void_p, c_void_p]),
    "amgt_spmm": (c_int, [c_int, c_double, P(AmgtBsr), c_int, c_void_p, c_int, c_double, c_void_p, c_int, c_void_p]),
    "amgt_spmm_rm": (c_int, [c_int, c_int, c_double, P(AmgtBsr), c_int, c_void_p, c_double, c_void_p, c_void_p]),
    "amgt_autotune": (c_int, [P(AmgtBsr), c_int, c_int, P(AmgtTuneResult), c_void_p]),
    "amgt_autotune_clear": (c_int, []),
    "amgt_bsr_l1_norms": (c_int, [P(AmgtBsr), c_void_p, c_void_p]),
    "amgt_bsr_residual": (c_int, [c_int, P(AmgtBsr), c_void_p, c_void_p, c_void_p, c_void_p]),
    "amgt_bsr_jacobi": (c_int, [c_int, P(AmgtBsr), c_void_p, c_double, c_void_p, c_void_p, c_void_p, c_void_p]),
    "amgt_bsr_pack": (c_int, [P(AmgtBsr), c_int, P(AmgtPbsr), c_void_p]),
    "amgt_pbsr_free": (c_int, [P(AmgtPbsr), c_void_p]),
    "amgt_pbsr_spmv": (c_int, [c_double, P(AmgtPbsr), c_void_p, c_double, c_void_p, c_void_p]),
    "amgt_pbsr_residual": (c_int, [P(AmgtPbsr), c_void_p, c_void_p, c_void_p, c_void_p]),
    "amgt_pbsr_jacobi": (c_int, [P(AmgtPbsr), c_void_p, c_double, c_void_p, c_void_p, c_void_p, c_void_p]),
    "amgt_spmv_segmented_noalloc": (c_int, [c_int, c_double, P(AmgtBsr), c_void_p, c_double, c_void_p, c_void_p]),
    "amgt_spgemm": (c_int, [c_int, P(AmgtBsr), P(AmgtBsr), P(AmgtBsr), P(AmgtCsr), c_void_p]),
    "amgt_spgemm_set_engine": (c_int, [c_int]),
    "amgt_amg_default_params": (None, [P(AmgtAmgParams)]),
    "amgt_amg_setup": (c_int, [P(AmgtCsr), c_int, P(AmgtCsr), P(AmgtAmgParams), P(c_void_p), c_void_p]),
    "amgt_amg_solve": (c_int, [c_void_p, c_void_p, c_void_p, P(c_int), P(c_double), c_void_p]),
    "amgt_amg_solve_multi": (c_int, [c_void_p, c_int, c_void_p, c_void_p, P(c_int), P(c_double), c_void_p]),
    "amgt_batch_setup": (c_int, [c_int, P(AmgtCsr), P(c_int), P(AmgtCsr), P(AmgtAmgParams), P(c_void_p), c_void_p]),
    "amgt_amg_solve_batch": (c_int, [c_void_p, c_void_p, c_void_p, P(c_int), P(c_double), P(c_int), c_void_p]),
    "amgt_batch_offsets": (c_int, [c_void_p, P(c_int), c_int]),
    "amgt_amg_num_levels": (c_int, [c_void_p]),
    "amgt_amg_level": (c_int, [c_void_p, c_int, P(AmgtBsr), P(c_int)]),
    "amgt_amg_setup_times": (c_int, [c_void_p, P(c_double)]),
    "amgt_amg_residual_history": (c_int, [c_void_p, P(c_double), c_int]),
    "amgt_amg_destroy": (c_int, [c_void_p, c_void_p]),
    "amgt_amg_setup_adaptive": (c_int, [P(AmgtCsr), c_void_p, c_void_p, P(AmgtAmgParams), P(c_void_p), c_void_p]),
    "amgt_boomer_default_params": (None, [P(AmgtBoomerParams)]),
    "amgt_boomer_coarsen_host": (c_int, [c_int, c_void_p, c_void_p, c_void_p, P(AmgtBoomerParams), c_void_p,
                                         P(AmgtCsr)]),
    "amgt_boomer_free_host": (c_int, [P(AmgtCsr)]),
    "amgt_boomer_interp": (c_int, [P(AmgtBsr), P(AmgtBoomerParams), P(AmgtCsr), c_void_p, c_void_p]),
    "amgt_boomer_hierarchy_host": (c_int, [c_int, c_void_p, c_void_p, c_void_p, P(AmgtBoomerParams), c_int, c_int,
                                           P(c_void_p)]),
    "amgt_boomer_hierarchy_levels": (c_int, [c_void_p]),
    "amgt_boomer_hierarchy_level": (c_int, [c_void_p, c_int, P(AmgtCsr), P(AmgtCsr)]),
    "amgt_boomer_hierarchy_free": (None, [c_void_p]),
    "amgt_level_features": (c_int, [P(AmgtBsr), c_int, P(c_int), P(ctypes.c_float), c_void_p]),
    "amgt_structured_interp": (c_int, [P(c_int), P(c_int), P(AmgtCsr), P(c_int), c_void_p]),
    "amgt_aniso_problem": (c_int, [P(c_int), c_double, c_double, P(AmgtCsr), c_void_p]),
    "amgt_mlp_forward": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "amgt_mlp_grad": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "amgt_mlp_train": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_int, c_int, ctypes.c_float, ctypes.c_uint,
                               P(ctypes.c_float), c_void_p]),
    "amgt_CSRMatrixCreate": (P(AmgtCSRMatrix), [c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_int]),
    "amgt_CSRMatrixDestroy": (c_int, [P(AmgtCSRMatrix)]),
    "amgt_set_stream": (c_int, [c_void_p]),
    "amgt_CSRSpGemm": (c_int, [P(AmgtCSRMatrix), P(AmgtCSRMatrix), P(P(AmgtCSRMatrix))]),
    "amgt_CSRMatrixMatvec": (c_int, [c_int, c_double, P(AmgtCSRMatrix), P(AmgtVector), c_double, P(AmgtVector),
                                     c_int]),
}

_lib = None


class AmgtError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = "?"
        if _lib is not None:
            msg = _lib.amgt_status_string(status).decode()
        super().__init__(f"{where} failed: {STATUS.get(status, status)} ({msg})")
        self.status = status


def lib():
    """The loaded library (raises when libamgt_b200.so is absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python amgt_b200/build.py` "
                              "(there is no fallback implementation)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str) -> None:
    if status != AMGT_OK:
        raise AmgtError(status, where)
