"""Python face of the AMG setup + solve (amgt_amg_* in include/amgt_b200.h).

The hierarchy, cycle and PCG run in libamgt_b200.so; the interpolation
operators come from the caller (HYPRE's coarsening and interpolation are
outside the AmgT path; amgt_b200.problems.interp gives linear interpolation
for structured grids).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib as L
from ._lib import AmgtAmgParams, AmgtBsr, check
from .mbsr import _stream, csr_struct


def default_params(**kw) -> AmgtAmgParams:
    p = AmgtAmgParams()
    L.lib().amgt_amg_default_params(ctypes.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


class AmgSolver:
    """A (n x n device CSR) and P_0..P_{L-2} (device CSR) -> hierarchy."""

    def __init__(self, A, Ps, params: AmgtAmgParams | None = None, stream=None):
        m, n, ia, ja, a = A
        self._keep = [A] + list(Ps)
        self._A = csr_struct(m, n, ia, ja, a)
        arr = (L.AmgtCsr * max(1, len(Ps)))()
        for i, (pm, pn, pia, pja, pa) in enumerate(Ps):
            arr[i] = csr_struct(pm, pn, pia, pja, pa)
        self.params = params if params is not None else default_params()
        self.h = ctypes.c_void_p()
        check(L.lib().amgt_amg_setup(ctypes.byref(self._A), len(Ps), arr, ctypes.byref(self.params),
                                     ctypes.byref(self.h), _stream(stream)), "amgt_amg_setup")
        self.n = m

    def solve(self, b: torch.Tensor, x: torch.Tensor | None = None, stream=None):
        """Solves A x = b (x: initial guess, updated in place); returns
        (x, iterations, relative residual)."""
        if x is None:
            x = torch.zeros_like(b)
        for v in (b, x):
            if not (v.is_cuda and v.dtype == torch.float64 and v.is_contiguous() and v.numel() == self.n):
                raise TypeError("b and x must be contiguous float64 CUDA vectors of the operator's size")
        it = ctypes.c_int()
        rel = ctypes.c_double()
        check(L.lib().amgt_amg_solve(self.h, b.data_ptr(), x.data_ptr(), ctypes.byref(it), ctypes.byref(rel),
                                     _stream(stream)), "amgt_amg_solve")
        return x, it.value, rel.value

    def solve_multi(self, B: torch.Tensor, X: torch.Tensor | None = None, stream=None):
        """Solves A X = B for the columns of B, (n, nrhs) row-major float64,
        nrhs <= 32, all at once (amgt_amg_solve_multi); returns (X,
        iterations per column, relative residual per column)."""
        n, nv = B.shape
        if X is None:
            X = torch.zeros_like(B)
        for T in (B, X):
            if not (T.is_cuda and T.dtype == torch.float64 and T.is_contiguous() and T.shape == (self.n, nv)):
                raise TypeError("B and X must be contiguous (n, nrhs) float64 CUDA tensors")
        its = (ctypes.c_int * nv)()
        rel = (ctypes.c_double * nv)()
        check(L.lib().amgt_amg_solve_multi(self.h, nv, B.data_ptr(), X.data_ptr(), its, rel, _stream(stream)),
              "amgt_amg_solve_multi")
        return X, list(its), list(rel)

    def num_levels(self) -> int:
        return L.lib().amgt_amg_num_levels(self.h)

    def level(self, l: int):
        """(rows, blocks, csr nonzeros, cycle precision) of level l."""
        b = AmgtBsr()
        prec = ctypes.c_int()
        check(L.lib().amgt_amg_level(self.h, l, ctypes.byref(b), ctypes.byref(prec)), "amgt_amg_level")
        return {"rows": b.row, "blocks": b.blc_num, "nnz": b.csr_nnz, "prec": prec.value}

    def level_csr(self, l: int):
        """Level l's operator as it is stored on the GPU, copied to a host
        scipy CSR (columns ascending)."""
        import scipy.sparse as sp

        from .mbsr import view

        b = AmgtBsr()
        prec = ctypes.c_int()
        check(L.lib().amgt_amg_level(self.h, l, ctypes.byref(b), ctypes.byref(prec)), "amgt_amg_level")
        c = L.AmgtCsr()
        check(L.lib().amgt_bsr_to_csr(ctypes.byref(b), ctypes.byref(c), None), "amgt_bsr_to_csr")
        shape = (c.num_rows, c.num_cols)
        try:
            ia = view(c.i, c.num_rows + 1, torch.int32).cpu().numpy()
            ja = view(c.j, c.num_nonzeros, torch.int32).cpu().numpy()
            a = view(c.data, c.num_nonzeros, torch.float64).cpu().numpy()
        finally:
            L.lib().amgt_csr_free(ctypes.byref(c), None)
        return sp.csr_matrix((a, ja, ia), shape=shape)

    def setup_times(self):
        ms = (ctypes.c_double * 4)()
        check(L.lib().amgt_amg_setup_times(self.h, ms), "amgt_amg_setup_times")
        return {"convert_A": ms[0], "convert_P_transpose": ms[1], "galerkin_spgemm": ms[2], "smoother_coarse": ms[3]}

    def history(self):
        n = L.lib().amgt_amg_residual_history(self.h, None, 0)
        buf = (ctypes.c_double * max(n, 1))()
        L.lib().amgt_amg_residual_history(self.h, buf, n)
        return list(buf[:n])

    def free(self, stream=None):
        if self.h:
            L.lib().amgt_amg_destroy(self.h, _stream(stream))
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class BatchSolver(AmgSolver):
    """Independent systems of uneven size, solved at once: systems = [(A,
    [P_0, ...]), ...] with device CSR tuples (amgt_batch_setup)."""

    def __init__(self, systems, params: AmgtAmgParams | None = None, stream=None):
        self._keep = [A for A, _ in systems] + [P for _, Ps in systems for P in Ps]
        ns = len(systems)
        A_arr = (L.AmgtCsr * ns)()
        nlev = (ctypes.c_int * ns)()
        flat = [P for _, Ps in systems for P in Ps]
        P_arr = (L.AmgtCsr * max(1, len(flat)))()
        for i, (A, Ps) in enumerate(systems):
            A_arr[i] = csr_struct(*A)
            nlev[i] = len(Ps)
        for i, P in enumerate(flat):
            P_arr[i] = csr_struct(*P)
        self.params = params if params is not None else default_params()
        self.h = ctypes.c_void_p()
        check(L.lib().amgt_batch_setup(ns, A_arr, nlev, P_arr, ctypes.byref(self.params), ctypes.byref(self.h),
                                       _stream(stream)), "amgt_batch_setup")
        offs = (ctypes.c_int * (ns + 1))()
        L.lib().amgt_batch_offsets(self.h, offs, ns + 1)
        self.offsets = list(offs)
        self.nsys = ns
        self.n = self.offsets[-1]

    def solve_batch(self, b: torch.Tensor, x: torch.Tensor | None = None, stream=None):
        """b, x: concatenated float64 CUDA vectors; returns (x, iterations
        per system, relative residual per system, loop iterations)."""
        if x is None:
            x = torch.zeros_like(b)
        for v in (b, x):
            if not (v.is_cuda and v.dtype == torch.float64 and v.is_contiguous() and v.numel() == self.n):
                raise TypeError("b and x must be contiguous float64 CUDA vectors of the batch's size")
        its = (ctypes.c_int * self.nsys)()
        rel = (ctypes.c_double * self.nsys)()
        bit = ctypes.c_int()
        check(L.lib().amgt_amg_solve_batch(self.h, b.data_ptr(), x.data_ptr(), its, rel, ctypes.byref(bit),
                                           _stream(stream)), "amgt_amg_solve_batch")
        return x, list(its), list(rel), bit.value
