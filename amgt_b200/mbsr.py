"""Python face of the mBSR C ABI over torch CUDA tensors.

torch is used for device memory and streams only; every operation runs a
kernel of libamgt_b200.so through ctypes.  Arrays the library allocates are
exposed as zero-copy torch views and freed with the owning object.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib as L
from ._lib import AmgtBsr, AmgtCsr, AmgtPbsr, check

DOUBLE, FLOAT, HALF, BF16 = L.DOUBLE, L.FLOAT, L.HALF, L.BF16
PREC_NAMES = {DOUBLE: "fp64", FLOAT: "fp32", HALF: "fp16", BF16: "bf16"}


def _stream(stream=None) -> int:
    s = torch.cuda.current_stream() if stream is None else stream
    return s.cuda_stream


class _DevArray:
    """__cuda_array_interface__ adapter for a raw device pointer."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def view(ptr, n: int, dtype: torch.dtype) -> torch.Tensor:
    """Zero-copy torch view of n elements at a library-owned device pointer."""
    typestr = {torch.int32: "<i4", torch.float64: "<f8", torch.float32: "<f4", torch.int16: "<i2",
               torch.uint16: "<u2"}[dtype]
    if not ptr or n == 0:
        return torch.empty(0, dtype=dtype, device="cuda")
    return torch.as_tensor(_DevArray(ptr, (n,), typestr), device="cuda")


def csr_struct(m: int, n: int, ia: torch.Tensor, ja: torch.Tensor, a: torch.Tensor) -> AmgtCsr:
    for t, dt in ((ia, torch.int32), (ja, torch.int32), (a, torch.float64)):
        if not (t.is_cuda and t.dtype == dt and t.is_contiguous()):
            raise TypeError("CSR arrays must be contiguous CUDA int32/int32/float64 tensors")
    return AmgtCsr(m, n, int(ja.numel()), ia.data_ptr(), ja.data_ptr(), a.data_ptr())


class Bsr:
    """An mBSR matrix owned by the library (amgt_bsr)."""

    def __init__(self):
        self.s = AmgtBsr()
        self._live = False

    # ---- construction
    @classmethod
    def from_csr(cls, m: int, n: int, ia: torch.Tensor, ja: torch.Tensor, a: torch.Tensor, stream=None) -> "Bsr":
        B = cls()
        c = csr_struct(m, n, ia, ja, a)
        check(L.lib().amgt_csr_to_bsr(ctypes.byref(c), ctypes.byref(B.s), _stream(stream)), "amgt_csr_to_bsr")
        B._live = True
        return B

    def free(self, stream=None) -> None:
        if self._live:
            L.lib().amgt_bsr_free(ctypes.byref(self.s), _stream(stream))
            self._live = False

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    # ---- properties
    @property
    def shape(self):
        return (self.s.row, self.s.col)

    @property
    def nblk(self) -> int:
        return self.s.blc_num

    def ptr(self) -> torch.Tensor:
        return view(self.s.blcPtr, self.s.blc_row + 1, torch.int32)

    def idx(self) -> torch.Tensor:
        return view(self.s.blcIdx, self.s.blc_num, torch.int32)

    def val(self) -> torch.Tensor:
        return view(self.s.blcVal, 16 * self.s.blc_num, torch.float64)

    def map(self) -> torch.Tensor:
        return view(self.s.blcMap, self.s.blc_num, torch.int16)

    def shadow(self, prec: int) -> torch.Tensor:
        n = 16 * self.s.blc_num
        if prec == FLOAT:
            return view(self.s.blcVal_fp32, n, torch.float32)
        p = self.s.blcVal_fp16 if prec == HALF else self.s.blcVal_bf16
        return view(p, n, torch.int16)

    def host(self) -> dict:
        """Copies of the arrays on the host (numpy), for checking."""
        import numpy as np

        torch.cuda.synchronize()
        return {"bptr": self.ptr().cpu().numpy(), "bidx": self.idx().cpu().numpy(),
                "bmap": self.map().cpu().numpy().view(np.uint16), "bval": self.val().cpu().numpy()}

    # ---- operations
    def make_shadow(self, prec: int, stream=None) -> None:
        check(L.lib().amgt_bsr_make_shadow(ctypes.byref(self.s), prec, _stream(stream)), "amgt_bsr_make_shadow")

    def make_exact(self, stream=None) -> int:
        """Exact narrow storage (amgt_bsr_make_exact); returns exact_prec."""
        check(L.lib().amgt_bsr_make_exact(ctypes.byref(self.s), _stream(stream)), "amgt_bsr_make_exact")
        return int(self.s.exact_prec)

    def balance(self, stream=None) -> None:
        check(L.lib().amgt_bsr_balance(ctypes.byref(self.s), _stream(stream)), "amgt_bsr_balance")

    def transpose(self, stream=None) -> "Bsr":
        T = Bsr()
        check(L.lib().amgt_bsr_transpose(ctypes.byref(self.s), ctypes.byref(T.s), _stream(stream)),
              "amgt_bsr_transpose")
        T._live = True
        return T

    def to_csr(self, stream=None):
        """(ia, ja, a) torch tensors (copies; the library arrays are freed)."""
        c = AmgtCsr()
        check(L.lib().amgt_bsr_to_csr(ctypes.byref(self.s), ctypes.byref(c), _stream(stream)), "amgt_bsr_to_csr")
        try:
            out = (view(c.i, c.num_rows + 1, torch.int32).clone(), view(c.j, c.num_nonzeros, torch.int32).clone(),
                   view(c.data, c.num_nonzeros, torch.float64).clone())
        finally:
            L.lib().amgt_csr_free(ctypes.byref(c), _stream(stream))
        return out

    def pack(self, prec: int = DOUBLE, stream=None) -> "PackedBsr":
        """Bitmap-packed copy of the values (the block structure stays
        borrowed from this matrix, which must outlive it)."""
        P_ = PackedBsr(self)
        check(L.lib().amgt_bsr_pack(ctypes.byref(self.s), prec, ctypes.byref(P_.s), _stream(stream)),
              "amgt_bsr_pack")
        P_._live = True
        return P_

    def spmv(self, x: torch.Tensor, y: torch.Tensor | None = None, alpha: float = 1.0, beta: float = 0.0,
             prec: int = DOUBLE, stream=None) -> torch.Tensor:
        if y is None:
            y = torch.zeros(self.s.row, dtype=torch.float64, device="cuda")
            beta = 0.0
        _vec_check(x, self.s.col)
        _vec_check(y, self.s.row)
        check(L.lib().amgt_spmv(prec, alpha, ctypes.byref(self.s), x.data_ptr(), beta, y.data_ptr(),
                                _stream(stream)), "amgt_spmv")
        return y

    def spmm(self, X: torch.Tensor, Y: torch.Tensor | None = None, alpha: float = 1.0, beta: float = 0.0,
             prec: int = DOUBLE, stream=None) -> torch.Tensor:
        """X, Y: (nvec, n) row-major tensors = column-major multivectors."""
        nvec = X.shape[0]
        if Y is None:
            Y = torch.zeros(nvec, self.s.row, dtype=torch.float64, device="cuda")
            beta = 0.0
        if not (X.is_cuda and X.dtype == torch.float64 and X.stride(1) == 1 and X.shape[1] == self.s.col):
            raise TypeError("X must be (nvec, ncols) float64 CUDA with unit inner stride")
        if not (Y.is_cuda and Y.dtype == torch.float64 and Y.stride(1) == 1 and Y.shape == (nvec, self.s.row)):
            raise TypeError("Y must be (nvec, nrows) float64 CUDA with unit inner stride")
        check(L.lib().amgt_spmm(prec, alpha, ctypes.byref(self.s), nvec, X.data_ptr(), X.stride(0), beta,
                                Y.data_ptr(), Y.stride(0), _stream(stream)), "amgt_spmm")
        return Y


    def spmm_rm(self, X: torch.Tensor, Y: torch.Tensor | None = None, alpha: float = 1.0, beta: float = 0.0,
                prec: int = DOUBLE, engine: int = 0, stream=None) -> torch.Tensor:
        """Row-major multivectors: X (ncols, nvec), Y (nrows, nvec), float64
        contiguous, nvec <= 32 (amgt_spmm_rm; engine 0 auto, 1 CUDA cores,
        2 tensor cores)."""
        nvec = X.shape[1]
        if Y is None:
            Y = torch.zeros(self.s.row, nvec, dtype=torch.float64, device="cuda")
            beta = 0.0
        for T, rows in ((X, self.s.col), (Y, self.s.row)):
            if not (T.is_cuda and T.dtype == torch.float64 and T.is_contiguous() and T.shape == (rows, nvec)):
                raise TypeError("X, Y must be contiguous (rows, nvec) float64 CUDA tensors")
        check(L.lib().amgt_spmm_rm(prec, engine, alpha, ctypes.byref(self.s), nvec, X.data_ptr(), beta,
                                   Y.data_ptr(), _stream(stream)), "amgt_spmm_rm")
        return Y

    def autotune(self, prec: int = DOUBLE, nvec: int = 1, stream=None) -> dict:
        """amgt_autotune: times the launch shapes on this matrix and keeps
        the fastest; returns {candidate code: ms} and the choice."""
        r = L.AmgtTuneResult()
        check(L.lib().amgt_autotune(ctypes.byref(self.s), prec, nvec, ctypes.byref(r), _stream(stream)),
              "amgt_autotune")
        return {"choice": r.choice, "ms": {int(r.candidate[i]): float(r.ms[i]) for i in range(r.count)}}


class PackedBsr:
    """amgt_pbsr: mBSR with only the set bits' values stored."""

    def __init__(self, owner: Bsr):
        self.s = AmgtPbsr()
        self._owner = owner
        self._live = False

    def free(self, stream=None) -> None:
        if self._live:
            L.lib().amgt_pbsr_free(ctypes.byref(self.s), _stream(stream))
            self._live = False

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def spmv(self, x, y=None, alpha=1.0, beta=0.0, stream=None):
        if y is None:
            y = torch.zeros(self.s.row, dtype=torch.float64, device="cuda")
            beta = 0.0
        _vec_check(x, self.s.col)
        _vec_check(y, self.s.row)
        check(L.lib().amgt_pbsr_spmv(alpha, ctypes.byref(self.s), x.data_ptr(), beta, y.data_ptr(),
                                     _stream(stream)), "amgt_pbsr_spmv")
        return y

    def residual(self, f, u, r=None, stream=None):
        r = torch.empty_like(f) if r is None else r
        check(L.lib().amgt_pbsr_residual(ctypes.byref(self.s), f.data_ptr(), u.data_ptr(), r.data_ptr(),
                                         _stream(stream)), "amgt_pbsr_residual")
        return r

    def jacobi(self, inv_l1, weight, f, u, out=None, stream=None):
        out = torch.empty_like(u) if out is None else out
        check(L.lib().amgt_pbsr_jacobi(ctypes.byref(self.s), inv_l1.data_ptr(), weight, f.data_ptr(),
                                       u.data_ptr(), out.data_ptr(), _stream(stream)), "amgt_pbsr_jacobi")
        return out


def _vec_check(v: torch.Tensor, n: int) -> None:
    if not (v.is_cuda and v.dtype == torch.float64 and v.is_contiguous() and v.numel() == n):
        raise TypeError(f"expected a contiguous float64 CUDA vector of {n} entries")


def spgemm(A: Bsr, B: Bsr, prec: int = DOUBLE, want_csr: bool = True, stream=None):
    """C = A*B.  Returns (C as Bsr, (ia, ja, a) views or None, csr owner)."""
    C = Bsr()
    c = AmgtCsr()
    check(L.lib().amgt_spgemm(prec, ctypes.byref(A.s), ctypes.byref(B.s), ctypes.byref(C.s),
                              ctypes.byref(c) if want_csr else None, _stream(stream)), "amgt_spgemm")
    C._live = True
    csr = None
    if want_csr:
        csr = CsrOwned(c)
    return C, csr


class CsrOwned:
    """A CSR matrix whose arrays the library allocated (amgt_csr)."""

    def __init__(self, c: AmgtCsr):
        self.s = c
        self._live = True

    @property
    def ia(self) -> torch.Tensor:
        return view(self.s.i, self.s.num_rows + 1, torch.int32)

    @property
    def ja(self) -> torch.Tensor:
        return view(self.s.j, self.s.num_nonzeros, torch.int32)

    @property
    def a(self) -> torch.Tensor:
        return view(self.s.data, self.s.num_nonzeros, torch.float64)

    def free(self, stream=None):
        if self._live:
            L.lib().amgt_csr_free(ctypes.byref(self.s), _stream(stream))
            self._live = False

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def kernel_launch_count() -> int:
    return int(L.lib().amgt_kernel_launch_count())


def init() -> None:
    check(L.lib().amgt_init(), "amgt_init")


def set_level_policy(precs) -> None:
    arr = (ctypes.c_int * len(precs))(*precs)
    check(L.lib().amgt_set_level_policy(arr, len(precs)), "amgt_set_level_policy")


def precision_for_level(level: int) -> int:
    return int(L.lib().amgt_precision_for_level(level))
