"""BoomerAMG's coarsening and interpolation (HMIS, strength threshold
theta, extended+i, P_max truncation) in front of the mBSR hierarchy.

BoomerSolver builds the hierarchy level by level through
amgt_amg_setup_adaptive: at each level the library hands over A_l, and
amgt_boomer_interp (host HMIS + ext+i, as HYPRE 2.31 runs HMIS on the host)
returns P_l; the Galerkin products, smoothers, coarse inverse and solve
are the library's GPU path.  Coarsening stops, as BoomerAMG's does, at a
level of at most max_coarse rows (HYPRE's default 9), or when a level does
not coarsen.  host_hierarchy() builds the same interpolation operators on
the CPU alone (Galerkin products by scipy), for callers and tests without a
GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from ._lib import AmgtAmgParams, AmgtBoomerParams, AmgtBsr, AmgtCsr, check


def params(theta: float = 0.25, max_row_sum: float = 1.0, p_max: int = 4, coarsen_type: int = 10) -> AmgtBoomerParams:
    """BoomerAMG settings: the ij driver's defaults (HMIS = coarsen type 10,
    theta 0.25, P_max 4, max_row_sum 1 = off); coarsen_type 8 is PMIS."""
    p = AmgtBoomerParams()
    L.lib().amgt_boomer_default_params(ctypes.byref(p))
    p.theta, p.max_row_sum, p.p_max, p.coarsen_type = theta, max_row_sum, p_max, coarsen_type
    return p


def diag_first(n, ia, ja, a):
    """Rows reordered: the diagonal first, the rest ascending (HYPRE's
    storage).  Rows must hold ascending columns; a row without a diagonal
    entry keeps its order."""
    ia = np.asarray(ia, np.int32)
    ja = np.asarray(ja, np.int32)
    a = np.asarray(a, np.float64)
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(ia))
    is_diag = ja == rows
    # an entry before its row's diagonal moves one place right; the diagonal
    # moves to the row's start
    before = np.zeros(ja.size, bool)
    dpos = np.full(n, -1, np.int64)
    dpos[rows[is_diag]] = np.flatnonzero(is_diag)
    has = dpos[rows] >= 0
    idx = np.arange(ja.size, dtype=np.int64)
    before[has] = idx[has] < dpos[rows[has]]
    dest = idx + before
    dest[is_diag] = ia[rows[is_diag]]
    ja2 = np.empty_like(ja)
    a2 = np.empty_like(a)
    ja2[dest] = ja
    a2[dest] = a
    return ia, ja2, a2


def coarsen_host(n, ia, ja, a, prm: AmgtBoomerParams | None = None):
    """One level on host arrays (rows diagonal first): (P as scipy CSR, C/F
    marker)."""
    import scipy.sparse as sp

    ia = np.ascontiguousarray(ia, np.int32)
    ja = np.ascontiguousarray(ja, np.int32)
    a = np.ascontiguousarray(a, np.float64)
    cf = np.zeros(n, np.int32)
    P = AmgtCsr()
    check(L.lib().amgt_boomer_coarsen_host(n, ia.ctypes.data, ja.ctypes.data, a.ctypes.data,
                                           ctypes.byref(prm) if prm is not None else None, cf.ctypes.data,
                                           ctypes.byref(P)), "amgt_boomer_coarsen_host")
    try:
        nnz = P.num_nonzeros
        pi = np.ctypeslib.as_array(ctypes.cast(P.i, ctypes.POINTER(ctypes.c_int)), (n + 1,)).copy()
        pj = np.ctypeslib.as_array(ctypes.cast(P.j, ctypes.POINTER(ctypes.c_int)), (max(nnz, 1),))[:nnz].copy()
        pa = np.ctypeslib.as_array(ctypes.cast(P.data, ctypes.POINTER(ctypes.c_double)), (max(nnz, 1),))[:nnz].copy()
        ncols = P.num_cols
    finally:
        L.lib().amgt_boomer_free_host(ctypes.byref(P))
    return sp.csr_matrix((pa, pj, pi), shape=(n, ncols)), cf


def hypre_hierarchy(A, prm: AmgtBoomerParams | None = None, max_coarse: int = 9, max_levels: int = 25):
    """The hierarchy as HYPRE's CPU BoomerAMG builds it on one process
    (amgt_boomer_hierarchy_host: coarsening, ext+i and truncation per level,
    Galerkin products in HYPRE's order and arithmetic).  A: scipy CSR whose
    rows become diagonal first, the rest ascending (the order of HYPRE's
    generators).  Returns ([P_0, ...], [A_0, A_1, ...]) as scipy CSR in
    HYPRE's stored column order."""
    import scipy.sparse as sp

    A = sp.csr_matrix(A)
    A.sort_indices()
    ia, ja, a = diag_first(A.shape[0], A.indptr, A.indices, A.data)
    lib = L.lib()
    h = ctypes.c_void_p()
    check(lib.amgt_boomer_hierarchy_host(A.shape[0], ia.ctypes.data, ja.ctypes.data, a.ctypes.data,
                                         ctypes.byref(prm if prm is not None else params()), max_levels, max_coarse,
                                         ctypes.byref(h)), "amgt_boomer_hierarchy_host")

    def copy(M):
        nz = M.num_nonzeros
        i = np.ctypeslib.as_array(ctypes.cast(M.i, ctypes.POINTER(ctypes.c_int)), (M.num_rows + 1,)).copy()
        if nz == 0:
            return sp.csr_matrix((np.zeros(0), np.zeros(0, np.int32), i), shape=(M.num_rows, M.num_cols))
        j = np.ctypeslib.as_array(ctypes.cast(M.j, ctypes.POINTER(ctypes.c_int)), (nz,)).copy()
        v = np.ctypeslib.as_array(ctypes.cast(M.data, ctypes.POINTER(ctypes.c_double)), (nz,)).copy()
        M2 = sp.csr_matrix((M.num_rows, M.num_cols))
        M2.data, M2.indices, M2.indptr = v, j, i  # keeps the stored column order
        return M2

    try:
        nl = lib.amgt_boomer_hierarchy_levels(h)
        Ps, As = [], []
        for l in range(nl):
            Am, Pm = AmgtCsr(), AmgtCsr()
            check(lib.amgt_boomer_hierarchy_level(h, l, ctypes.byref(Am), ctypes.byref(Pm)),
                  "amgt_boomer_hierarchy_level")
            As.append(copy(Am))
            if l < nl - 1:
                Ps.append(copy(Pm))
    finally:
        lib.amgt_boomer_hierarchy_free(h)
    return Ps, As


def ij_random_rhs(n: int, seed: int = 22775) -> np.ndarray:
    """The right-hand side of HYPRE's ij driver with -rhsrand
    (R/test/ij.c:3463-3466, hypre_SeqVectorSetRandomValues): 2 u - 1 per
    entry, u from Park and Miller's minimal standard generator seeded with
    `seed`, scaled to unit 2-norm.  The sequence is generated in blocks:
    s_{k+j} = (16807^j mod m) s_k mod m."""
    m, a = 2147483647, 16807
    blk = 1024
    first = np.empty(blk, np.int64)
    s = seed if 0 < seed < m else (1 if seed < 1 else m - 1)
    for k in range(blk):
        s = (a * s) % m
        first[k] = s
    step = pow(a, blk, m)
    nb = (n + blk - 1) // blk
    out = np.empty(nb * blk, np.int64)
    cur = first
    for b in range(nb):
        out[b * blk:(b + 1) * blk] = cur
        cur = (cur * step) % m
    v = 2.0 * (out[:n].astype(np.float64) / float(m)) - 1.0
    return v / np.sqrt(np.dot(v, v))


def host_hierarchy(A, prm: AmgtBoomerParams | None = None, max_coarse: int = 9, max_levels: int = 25):
    """The hierarchy BoomerSolver builds, restated on the CPU: each level's
    operator (scipy's Galerkin product) sorted and stored diagonal first,
    as amgt_boomer_interp receives it from the GPU, then coarsened by
    amgt_boomer_coarsen_host.  A: scipy CSR; returns ([P_0, ...],
    [A_0, A_1, ...])."""
    import scipy.sparse as sp

    As, Ps = [sp.csr_matrix(A)], []
    while As[-1].shape[0] > max_coarse and len(As) < max_levels:
        Al = As[-1]
        Al.sort_indices()
        ia, ja, a = diag_first(Al.shape[0], Al.indptr, Al.indices, Al.data)
        P, _ = coarsen_host(Al.shape[0], ia, ja, a, prm)
        if P.shape[1] == 0 or P.shape[1] >= Al.shape[0]:
            break
        Ps.append(P)
        As.append(sp.csr_matrix(P.T @ Al @ P))
    return Ps, As


COARSEN_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_int, ctypes.POINTER(AmgtBsr), ctypes.POINTER(AmgtCsr),
                              ctypes.POINTER(ctypes.c_int), ctypes.c_void_p)


def _solver_class():
    import torch

    from .amg import AmgSolver, default_params
    from .mbsr import _stream, csr_struct

    class BoomerSolver(AmgSolver):
        """The GPU hierarchy with BoomerAMG's coarsening and interpolation.

        levels="hypre" (default): the interpolation operators of HYPRE's
        own host setup (hypre_hierarchy on a host copy of A), uploaded once;
        the library forms the Galerkin products, smoothers and coarse solve
        (amgt_amg_setup).  The hierarchy is the one HYPRE's CPU BoomerAMG
        builds for the same matrix.
        levels="device": level by level from the GPU's own Galerkin
        products (amgt_boomer_interp in the callback of
        amgt_amg_setup_adaptive): each A_l is copied to the host, sorted
        and stored diagonal first, coarsened, and P_l uploaded.

        A: device CSR tuple (m, n, ia, ja, a).  precs[l]: level l's
        precision in the device mode (the last entry for deeper levels);
        the hypre mode follows the level policy (amgt_set_level_policy).
        host_setup_s: seconds of host coarsening (hypre mode).  trace: rows
        and coarse rows per level."""

        def __init__(self, A, prm: AmgtBoomerParams | None = None, amg_params: AmgtAmgParams | None = None,
                     precs=(L.DOUBLE,), max_coarse: int = 9, max_levels: int = 25, levels: str = "hypre",
                     stream=None):
            import time

            import scipy.sparse as sp

            self.bparams = prm if prm is not None else params()
            if levels == "hypre":
                m, n, ia, ja, a = A
                Ah = sp.csr_matrix((a.cpu().numpy(), ja.cpu().numpy(), ia.cpu().numpy()), shape=(m, n))
                t0 = time.perf_counter()
                Ps, As = hypre_hierarchy(Ah, self.bparams, max_coarse=max_coarse, max_levels=max_levels)
                self.host_setup_s = time.perf_counter() - t0
                self.trace = [{"level": l, "rows": int(As[l].shape[0]),
                               "coarse": int(As[l + 1].shape[0]) if l + 1 < len(As) else None}
                              for l in range(len(As))]
                dev = a.device
                for P in Ps:  # same operator; sorted rows take the conversion's merge path
                    P.sort_indices()
                Pd = [(P.shape[0], P.shape[1], torch.from_numpy(P.indptr.astype(np.int32)).to(dev),
                       torch.from_numpy(P.indices.astype(np.int32)).to(dev), torch.from_numpy(P.data).to(dev))
                      for P in Ps]
                super().__init__(A, Pd, amg_params, stream=stream)
                return
            if levels != "device":
                raise ValueError("levels must be 'hypre' or 'device'")
            m, n, ia, ja, a = A
            self._keep = [A]
            self._A = csr_struct(m, n, ia, ja, a)
            self.params = amg_params if amg_params is not None else default_params()
            self.host_setup_s = None
            self.trace = []
            Ps, state = [], {"err": None}

            def cb(level, Ap, Pp, precp, ctx):
                try:
                    Al = Ap.contents
                    precp[0] = int(precs[min(level, len(precs) - 1)])
                    if Al.row <= max_coarse or level + 1 >= max_levels:
                        self.trace.append({"level": level, "rows": int(Al.row), "coarse": None})
                        return 1
                    P = AmgtCsr()
                    check(L.lib().amgt_boomer_interp(ctypes.byref(Al), ctypes.byref(self.bparams), ctypes.byref(P),
                                                     None, _stream(stream)), "amgt_boomer_interp")
                    Ps.append(P)
                    self.trace.append({"level": level, "rows": int(Al.row), "coarse": int(P.num_cols)})
                    if P.num_cols == 0 or P.num_cols >= Al.row:
                        return 1  # no coarsening: this level is the coarsest
                    Pp[0] = P
                    return 0
                except Exception as e:  # noqa: BLE001 - reported after the setup returns
                    state["err"] = e
                    return -1

            fn = COARSEN_FN(cb)
            self.h = ctypes.c_void_p()
            try:
                rc = L.lib().amgt_amg_setup_adaptive(ctypes.byref(self._A), ctypes.cast(fn, ctypes.c_void_p), None,
                                                     ctypes.byref(self.params), ctypes.byref(self.h),
                                                     _stream(stream))
            finally:
                for P in Ps:
                    L.lib().amgt_csr_free(ctypes.byref(P), _stream(stream))
            if state["err"] is not None:
                raise state["err"]
            check(rc, "amgt_amg_setup_adaptive")
            self.n = m

        def operator_complexity(self) -> float:
            nnz = [self.level(l)["nnz"] for l in range(self.num_levels())]
            return sum(nnz) / nnz[0]

    return BoomerSolver


def BoomerSolver(*args, **kw):  # noqa: N802 - a class factory keeps torch out of host-only imports
    return _solver_class()(*args, **kw)
