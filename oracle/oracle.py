"""TEST INFRASTRUCTURE ONLY: numpy front end of the C oracle.

The oracle is a CPU restatement of AmgT's mBSR path (``amgt_oracle.c``).
Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product (``amgt_b200``) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libamgt_oracle.so")
_lib = None

DOUBLE, FLOAT, HALF, BF16 = 0, 1, 2, 3

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(dtype=np.uint16, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64


def build() -> str:
    """Compile the oracle with its Makefile (gcc); returns the .so path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "amgt_oracle.c")
        ):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        c_int, c_double = ctypes.c_int, ctypes.c_double
        L.orc_num_threads.restype = c_int
        L.orc_set_num_threads.argtypes = [c_int]
        L.orc_rand_uniform.argtypes = [ctypes.c_uint64, _i64, _f64p]
        L.orc_gen_laplacian.restype = _i64
        L.orc_gen_laplacian.argtypes = [c_int, c_int, c_int, c_double, c_double, c_double, _i32p, _i32p, _f64p]
        L.orc_gen_box.restype = _i64
        L.orc_gen_box.argtypes = [c_int, c_int, c_int, _i32p, _i32p, _f64p]
        L.orc_gen_varcoef27.restype = _i64
        L.orc_gen_varcoef27.argtypes = [c_int, c_int, c_int, ctypes.c_uint64, c_double, c_double, _i32p, _i32p, _f64p]
        L.orc_gen_interp.restype = _i64
        L.orc_gen_interp.argtypes = [c_int, c_int, c_int, _i32p, _i32p, _f64p,
                                     ctypes.POINTER(c_int), ctypes.POINTER(c_int), ctypes.POINTER(c_int)]
        L.orc_to_half.restype = ctypes.c_uint16
        L.orc_to_half.argtypes = [c_double]
        L.orc_to_bf16.restype = ctypes.c_uint16
        L.orc_to_bf16.argtypes = [c_double]
        L.orc_make_shadow.argtypes = [c_int, _i64, _f64p, _vp]
        L.orc_csr2bsr_count.restype = _i64
        L.orc_csr2bsr_count.argtypes = [c_int, c_int, _i32p, _i32p, _i32p, ctypes.POINTER(c_int)]
        L.orc_csr2bsr_fill.argtypes = [c_int, c_int, _i32p, _i32p, _vp, _i32p, _i32p, _u16p, _vp,
                                       ctypes.POINTER(c_double), ctypes.POINTER(c_double)]
        L.orc_bsr2csr_count.restype = _i64
        L.orc_bsr2csr_count.argtypes = [c_int, _i32p, _u16p, _i32p]
        L.orc_bsr2csr_fill.argtypes = [c_int, _i32p, _i32p, _u16p, _vp, _i32p, _i32p, _vp]
        L.orc_bsr_spmv.argtypes = [c_int, c_int, c_int, _i32p, _i32p, _f64p, c_double, _f64p, c_double, _f64p]
        L.orc_bsr_spmv_absbound.argtypes = [c_int, c_int, _i32p, _i32p, _f64p, c_double, _f64p, c_double, _f64p, _f64p]
        L.orc_bitmatmul.restype = ctypes.c_uint16
        L.orc_bitmatmul.argtypes = [ctypes.c_uint16, ctypes.c_uint16]
        L.orc_spgemm_count.restype = _i64
        L.orc_spgemm_count.argtypes = [c_int, _i32p, _i32p, _u16p, c_int, _i32p, _i32p, _u16p, _vp,
                                       ctypes.POINTER(_i64)]
        L.orc_spgemm_fill.argtypes = [c_int, c_int, _i32p, _i32p, _u16p, _f64p, c_int, _i32p, _i32p, _u16p,
                                      _f64p, _i32p, _i32p, _u16p, _f64p, _vp]
        L.orc_spgemm_fill_fma.argtypes = [c_int, c_int, _i32p, _i32p, _u16p, _f64p, c_int, _i32p, _i32p, _u16p,
                                      _f64p, _i32p, _i32p, _u16p, _f64p, _vp]
        L.orc_amg_setup.restype = _vp
        L.orc_amg_setup.argtypes = [c_int, _i32p, _i32p, _f64p, c_int, _vp, _vp, _vp, _vp, _vp, c_double]
        L.orc_amg_solve.restype = c_int
        L.orc_amg_solve.argtypes = [_vp, _f64p, _f64p, c_double, c_int, _f64p, ctypes.POINTER(c_double)]
        L.orc_amg_num_levels.restype = c_int
        L.orc_amg_num_levels.argtypes = [_vp]
        L.orc_amg_level_size.restype = c_int
        L.orc_amg_level_size.argtypes = [_vp, c_int, ctypes.POINTER(c_int)]
        L.orc_amg_free.argtypes = [_vp]
        L.orc_bsr_transpose.argtypes = [c_int, c_int, _i32p, _i32p, _u16p, _vp, _i32p, _i32p, _u16p, _vp]
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def num_threads() -> int:
    return lib().orc_num_threads()


# ------------------------------------------------------------------ formats
@dataclass
class CSR:
    m: int
    n: int
    ia: np.ndarray  # int32 [m+1]
    ja: np.ndarray  # int32 [nnz]
    a: np.ndarray  # float64 [nnz]

    @property
    def nnz(self) -> int:
        return int(self.ia[-1])

    def to_scipy(self):
        import scipy.sparse as sp

        return sp.csr_matrix((self.a, self.ja, self.ia), shape=(self.m, self.n))


@dataclass
class BSR:
    m: int
    n: int
    bptr: np.ndarray  # int32 [brow+1]
    bidx: np.ndarray  # int32 [nblk]
    bmap: np.ndarray  # uint16 [nblk]
    bval: np.ndarray | None  # float64 [nblk*16]
    stand: float = 0.0
    avg_nnz: float = 0.0
    max_row: int = 0

    @property
    def brow(self) -> int:
        return (self.m + 3) // 4

    @property
    def bcol(self) -> int:
        return (self.n + 3) // 4

    @property
    def nblk(self) -> int:
        return int(self.bptr[-1])


# --------------------------------------------------------------- generators
def laplacian(nx: int, ny: int, nz: int, cx=1.0, cy=1.0, cz=1.0) -> CSR:
    n = nx * ny * nz
    ia = np.zeros(n + 1, np.int32)
    ja = np.zeros(n * 7, np.int32)
    a = np.zeros(n * 7, np.float64)
    nnz = lib().orc_gen_laplacian(nx, ny, nz, cx, cy, cz, ia, ja, a)
    return CSR(n, n, ia, ja[:nnz].copy(), a[:nnz].copy())


def box(nx: int, ny: int, nz: int) -> CSR:
    """27-point (3D) / 9-point (2D) Laplacian."""
    n = nx * ny * nz
    st = 27 if nz > 1 else 9
    ia = np.zeros(n + 1, np.int32)
    ja = np.zeros(n * st, np.int32)
    a = np.zeros(n * st, np.float64)
    nnz = lib().orc_gen_box(nx, ny, nz, ia, ja, a)
    return CSR(n, n, ia, ja[:nnz].copy(), a[:nnz].copy())


def varcoef27(nx: int, ny: int, nz: int, seed: int = 1, sigma: float = 2.0, ratio: float = 1e3) -> CSR:
    n = nx * ny * nz
    ia = np.zeros(n + 1, np.int32)
    ja = np.zeros(n * 27, np.int32)
    a = np.zeros(n * 27, np.float64)
    nnz = lib().orc_gen_varcoef27(nx, ny, nz, seed, sigma, ratio, ia, ja, a)
    return CSR(n, n, ia, ja[:nnz].copy(), a[:nnz].copy())


def interp(nx: int, ny: int, nz: int):
    """Linear interpolation P (fine x coarse) and the coarse grid dims."""
    n = nx * ny * nz
    ia = np.zeros(n + 1, np.int32)
    ja = np.zeros(n * 8, np.int32)
    a = np.zeros(n * 8, np.float64)
    c = [ctypes.c_int(), ctypes.c_int(), ctypes.c_int()]
    nnz = lib().orc_gen_interp(nx, ny, nz, ia, ja, a, *[ctypes.byref(v) for v in c])
    cd = tuple(v.value for v in c)
    nc = cd[0] * cd[1] * cd[2]
    return CSR(n, nc, ia, ja[:nnz].copy(), a[:nnz].copy()), cd


def rand_uniform(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, np.float64)
    lib().orc_rand_uniform(seed, n, out)
    return out


# ---------------------------------------------------------------- rounding
def make_shadow(prec: int, vals: np.ndarray) -> np.ndarray:
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    out = np.empty(vals.size, np.float32 if prec == FLOAT else np.uint16)
    lib().orc_make_shadow(prec, vals.size, vals, out.ctypes.data)
    return out


def to_half_bits(d: float) -> int:
    return int(lib().orc_to_half(float(d)))


def to_bf16_bits(d: float) -> int:
    return int(lib().orc_to_bf16(float(d)))


# ---------------------------------------------------------------- kernels
def csr2bsr(A: CSR, values: bool = True) -> BSR:
    L = lib()
    brow = (A.m + 3) // 4
    bptr = np.zeros(brow + 1, np.int32)
    mx = ctypes.c_int()
    nb = L.orc_csr2bsr_count(A.m, A.n, A.ia, A.ja, bptr, ctypes.byref(mx))
    bidx = np.zeros(max(nb, 1), np.int32)
    bmap = np.zeros(max(nb, 1), np.uint16)
    bval = np.zeros(max(nb, 1) * 16, np.float64) if values else None
    st, av = ctypes.c_double(), ctypes.c_double()
    L.orc_csr2bsr_fill(A.m, A.n, A.ia, A.ja, A.a.ctypes.data if values else None, bptr, bidx, bmap,
                       bval.ctypes.data if values else None, ctypes.byref(st), ctypes.byref(av))
    return BSR(A.m, A.n, bptr, bidx[:nb], bmap[:nb], None if bval is None else bval[: nb * 16],
               st.value, av.value, mx.value)


def bsr2csr(B: BSR, values: bool = True) -> CSR:
    L = lib()
    ia = np.zeros(B.m + 1, np.int32)
    nnz = L.orc_bsr2csr_count(B.m, B.bptr, np.ascontiguousarray(B.bmap), ia)
    ja = np.zeros(max(nnz, 1), np.int32)
    a = np.zeros(max(nnz, 1), np.float64)
    L.orc_bsr2csr_fill(B.m, B.bptr, np.ascontiguousarray(B.bidx), np.ascontiguousarray(B.bmap),
                       B.bval.ctypes.data if (values and B.bval is not None) else None, ia, ja,
                       a.ctypes.data if values else None)
    return CSR(B.m, B.n, ia, ja[:nnz], a[:nnz])


def spmv(B: BSR, x: np.ndarray, y: np.ndarray | None = None, alpha=1.0, beta=0.0, prec=DOUBLE) -> np.ndarray:
    y = np.zeros(B.m) if y is None else np.array(y, dtype=np.float64, copy=True)
    lib().orc_bsr_spmv(prec, B.m, B.n, B.bptr, B.bidx, B.bval, alpha, np.ascontiguousarray(x, np.float64),
                       beta, y)
    return y


def spmv_bound(B: BSR, x: np.ndarray, y: np.ndarray | None, alpha=1.0, beta=0.0) -> np.ndarray:
    y0 = np.zeros(B.m) if y is None else np.ascontiguousarray(y, np.float64)
    s = np.zeros(B.m)
    lib().orc_bsr_spmv_absbound(B.m, B.n, B.bptr, B.bidx, B.bval, alpha, np.ascontiguousarray(x, np.float64),
                                beta, y0, s)
    return s


def bitmatmul(a: int, b: int) -> int:
    return int(lib().orc_bitmatmul(a, b))


def spgemm_count(A: BSR, B: BSR):
    """(C blocks, C CSR nonzeros) without values."""
    L = lib()
    bits = _i64()
    nb = L.orc_spgemm_count(A.brow, A.bptr, A.bidx, A.bmap, B.bcol, B.bptr, B.bidx, B.bmap, None,
                            ctypes.byref(bits))
    return int(nb), int(bits.value)


def spgemm(A: BSR, B: BSR, prec=DOUBLE, contract=True):
    """C = A*B in mBSR; returns (C, shadow or None).  contract (fp64): each
    4x4 product entry is the k-ordered fused multiply-add chain of the
    reference's fp64 kernel; False: separate multiply and add."""
    L = lib()
    cptr = np.zeros(A.brow + 1, np.int32)
    bits = _i64()
    nb = L.orc_spgemm_count(A.brow, A.bptr, A.bidx, A.bmap, B.bcol, B.bptr, B.bidx, B.bmap,
                            cptr.ctypes.data, ctypes.byref(bits))
    cidx = np.zeros(max(nb, 1), np.int32)
    cmap = np.zeros(max(nb, 1), np.uint16)
    cval = np.zeros(max(nb, 1) * 16, np.float64)
    sh = None
    if prec != DOUBLE:
        sh = np.zeros(max(nb, 1) * 16, np.float32 if prec == FLOAT else np.uint16)
    fill = L.orc_spgemm_fill_fma if contract else L.orc_spgemm_fill
    fill(prec, A.brow, A.bptr, A.bidx, A.bmap, A.bval, B.bcol, B.bptr, B.bidx, B.bmap, B.bval,
         cptr, cidx, cmap, cval, None if sh is None else sh.ctypes.data)
    C = BSR(A.m, B.n, cptr, cidx[:nb], cmap[:nb], cval[: nb * 16])
    return C, (None if sh is None else sh[: nb * 16])


def transpose(B: BSR) -> BSR:
    L = lib()
    tptr = np.zeros(B.bcol + 1, np.int32)
    nb = B.nblk
    tidx = np.zeros(max(nb, 1), np.int32)
    tmap = np.zeros(max(nb, 1), np.uint16)
    tval = np.zeros(max(nb, 1) * 16, np.float64)
    L.orc_bsr_transpose(B.brow, B.bcol, B.bptr, np.ascontiguousarray(B.bidx), np.ascontiguousarray(B.bmap),
                        None if B.bval is None else B.bval.ctypes.data, tptr, tidx, tmap, tval.ctypes.data)
    return BSR(B.n, B.m, tptr, tidx[:nb], tmap[:nb], tval[: nb * 16])


# --------------------------------------------------------------------- AMG
class Amg:
    """The oracle's AMG-PCG (fp64): Galerkin hierarchy on mBSR from given
    interpolation operators, V(1,1) l1-Jacobi, dense coarsest inverse."""

    def __init__(self, A: CSR, Ps, w: float = 1.0):
        L = lib()
        nP = len(Ps)
        self._keep = [A] + list(Ps)
        pm = np.array([P.m for P in Ps] or [0], np.int32)
        pn = np.array([P.n for P in Ps] or [0], np.int32)
        pia = (ctypes.c_void_p * max(nP, 1))(*[P.ia.ctypes.data for P in Ps])
        pja = (ctypes.c_void_p * max(nP, 1))(*[P.ja.ctypes.data for P in Ps])
        pa = (ctypes.c_void_p * max(nP, 1))(*[P.a.ctypes.data for P in Ps])
        self._arrs = (pm, pn, pia, pja, pa)
        self.h = L.orc_amg_setup(A.m, A.ia, A.ja, A.a, nP, pm.ctypes.data, pn.ctypes.data,
                                 ctypes.cast(pia, ctypes.c_void_p), ctypes.cast(pja, ctypes.c_void_p),
                                 ctypes.cast(pa, ctypes.c_void_p), w)
        self.n = A.m

    def solve(self, b, x0=None, tol=1e-8, maxit=200):
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        hist = np.zeros(maxit + 1)
        rel = ctypes.c_double()
        it = lib().orc_amg_solve(self.h, np.ascontiguousarray(b, np.float64), x, tol, maxit, hist, ctypes.byref(rel))
        return x, it, rel.value, hist[: it + 1]

    def levels(self):
        out = []
        for l in range(lib().orc_amg_num_levels(self.h)):
            nb = ctypes.c_int()
            n = lib().orc_amg_level_size(self.h, l, ctypes.byref(nb))
            out.append((n, nb.value))
        return out

    def __del__(self):
        try:
            lib().orc_amg_free(self.h)
        except Exception:
            pass


def geometric_hierarchy(nx, ny, nz, coarse_rows=64):
    """Linear interpolation operators from (nx, ny, nz) down to a grid of at
    most coarse_rows points."""
    Ps = []
    dims = (nx, ny, nz)
    while dims[0] * dims[1] * dims[2] > coarse_rows:
        P, cd = interp(*dims)
        if cd == dims:
            break
        Ps.append(P)
        dims = cd
    return Ps
