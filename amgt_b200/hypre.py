"""HYPRE-named mirror of the two AmgT hooks, for callers in Python.

    hypreDevice_CSRSpGemm(A, B) -> C
        AmgT_HYPRE/src/seq_mv/csr_spgemm_device.c:2579-2608
    hypre_CSRMatrixMatvecCusparseNewAPI(trans, alpha, A, x, beta, y, offset)
        AmgT_HYPRE/src/seq_mv/csr_matvec_device.c:2397-2437

Both go through the C mirror layer of libamgt_b200.so (amgt_CSRSpGemm,
amgt_CSRMatrixMatvec), which keeps HYPRE's semantics: lazy, cached CSR ->
mBSR conversion per matrix, precision chosen from the matrix's AMG level
(get_calculationPrecison), an SpGEMM result that owns its CSR arrays and
carries its mBSR, y = alpha*op(A)*x + beta*y with offset 0.
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib as L
from ._lib import AmgtCSRMatrix, AmgtVector, check
from .mbsr import _stream, view


def _set_stream(stream=None):
    L.lib().amgt_set_stream(_stream(stream))


class CSRMatrix:
    """Device CSR matrix with the AmgT fields of hypre_CSRMatrix
    (seq_mv.h:154-199): level tag, mBSR cache, transpose cache."""

    def __init__(self, handle, keep=()):
        self.h = handle
        self._keep = keep  # tensors whose memory the matrix borrows

    @classmethod
    def create(cls, num_rows: int, num_cols: int, ia: torch.Tensor, ja: torch.Tensor, a: torch.Tensor,
               level: int = 0) -> "CSRMatrix":
        for t, dt in ((ia, torch.int32), (ja, torch.int32), (a, torch.float64)):
            if not (t.is_cuda and t.dtype == dt and t.is_contiguous()):
                raise TypeError("CSR arrays must be contiguous CUDA int32/int32/float64 tensors")
        h = L.lib().amgt_CSRMatrixCreate(num_rows, num_cols, int(ja.numel()), ia.data_ptr(), ja.data_ptr(),
                                         a.data_ptr(), level)
        if not h:
            raise ValueError("amgt_CSRMatrixCreate rejected the sizes")
        return cls(h, (ia, ja, a))

    def destroy(self) -> None:
        if self.h:
            _set_stream()
            L.lib().amgt_CSRMatrixDestroy(self.h)
            self.h = None
            self._keep = ()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    @property
    def s(self) -> AmgtCSRMatrix:
        return self.h.contents

    num_rows = property(lambda self: self.s.csr.num_rows)
    num_cols = property(lambda self: self.s.csr.num_cols)
    num_nonzeros = property(lambda self: self.s.csr.num_nonzeros)
    bsr_tag = property(lambda self: ord(self.s.bsr_tag))
    owns_data = property(lambda self: ord(self.s.owns_data))

    @property
    def level(self) -> int:
        return self.s.coasen_level

    @level.setter
    def level(self, v: int) -> None:
        self.s.coasen_level = int(v)

    @property
    def i(self) -> torch.Tensor:
        return view(self.s.csr.i, self.num_rows + 1, torch.int32)

    @property
    def j(self) -> torch.Tensor:
        return view(self.s.csr.j, self.num_nonzeros, torch.int32)

    @property
    def data(self) -> torch.Tensor:
        return view(self.s.csr.data, self.num_nonzeros, torch.float64)

    @property
    def bsr(self):
        """The cached amgt_bsr struct (None before first use)."""
        return self.s.bsr_mat.contents if self.s.bsr_mat else None


def hypre_Level(A: CSRMatrix) -> int:
    return A.level


def hypreDevice_CSRSpGemm(A: CSRMatrix, B: CSRMatrix, stream=None) -> CSRMatrix:
    _set_stream(stream)
    out = ctypes.POINTER(AmgtCSRMatrix)()
    check(L.lib().amgt_CSRSpGemm(A.h, B.h, ctypes.byref(out)), "hypreDevice_CSRSpGemm")
    return CSRMatrix(out)


def _vector(t: torch.Tensor) -> AmgtVector:
    if not (t.is_cuda and t.dtype == torch.float64):
        raise TypeError("vectors must be float64 CUDA tensors")
    if t.dim() == 1:
        if not t.is_contiguous():
            raise TypeError("vector must be contiguous")
        return AmgtVector(t.data_ptr(), t.numel(), 1, t.numel())
    if t.dim() == 2 and t.stride(1) == 1:
        # (num_vectors, size) row-major == HYPRE's column-wise multivector storage
        return AmgtVector(t.data_ptr(), t.shape[1], t.shape[0], t.stride(0))
    raise TypeError("multivector must be (num_vectors, size) with unit inner stride")


def hypre_CSRMatrixMatvecCusparseNewAPI(trans: int, alpha: float, A: CSRMatrix, x: torch.Tensor, beta: float,
                                        y: torch.Tensor, offset: int = 0, stream=None) -> int:
    """y = alpha * op(A) * x + beta * y; returns 0 (raises on error)."""
    _set_stream(stream)
    xv, yv = _vector(x), _vector(y)
    check(L.lib().amgt_CSRMatrixMatvec(int(trans), float(alpha), A.h, ctypes.byref(xv), float(beta),
                                       ctypes.byref(yv), int(offset)), "hypre_CSRMatrixMatvecCusparseNewAPI")
    return 0
