"""GPU tests of the fused smoother / residual kernels and of the AMG
setup + solve, against the oracle.

Fused kernels: per row |out - out_oracle| <= 1e-12 * scale (fp64 sums in a
different fixed order).  Solve: the fp64 GPU path reproduces the oracle's
PCG: the same iteration count, a residual history equal to 1e-6 relative,
and a solution equal to 1e-9 relative.  Mixed precision: converges to
||b - A x|| / ||b|| <= 1e-8 checked in fp64 by the oracle, with its error
against the fp64 oracle solution reported."""
import numpy as np
import pytest
import torch

from gpu_util import to_dev

pytestmark = pytest.mark.gpu


def _bsr(amgt, A):
    return amgt.Bsr.from_csr(*to_dev(A))


def test_fused_residual_and_jacobi(amgt, orc):
    import ctypes

    L = amgt.lib()
    A = orc.varcoef27(15, 13, 11, seed=3)
    R = orc.csr2bsr(A)
    G = _bsr(amgt, A)
    u = orc.rand_uniform(1, A.n)
    f = orc.rand_uniform(2, A.n)
    S = A.to_scipy()
    l1 = np.asarray(abs(S).sum(axis=1)).ravel()
    ud, fd = torch.from_numpy(u).cuda(), torch.from_numpy(f).cuda()
    out = torch.zeros(A.m, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    # l1 norms
    l1d = torch.zeros(A.m, dtype=torch.float64, device="cuda")
    assert L.amgt_bsr_l1_norms(ctypes.byref(G.s), l1d.data_ptr(), st) == 0
    np.testing.assert_allclose(l1d.cpu().numpy(), l1, rtol=1e-14)
    # residual
    assert L.amgt_bsr_residual(0, ctypes.byref(G.s), fd.data_ptr(), ud.data_ptr(), out.data_ptr(), st) == 0
    want = f - orc.spmv(R, u)
    scale = orc.spmv_bound(R, u, f, alpha=-1.0, beta=1.0)
    assert np.all(np.abs(out.cpu().numpy() - want) <= 1e-12 * scale)
    # one l1-Jacobi sweep, weight 0.8
    inv = torch.from_numpy(1.0 / l1).cuda()
    assert L.amgt_bsr_jacobi(0, ctypes.byref(G.s), inv.data_ptr(), 0.8, fd.data_ptr(), ud.data_ptr(),
                             out.data_ptr(), st) == 0
    want = u + 0.8 * (f - orc.spmv(R, u)) / l1
    assert np.all(np.abs(out.cpu().numpy() - want) <= 1e-12 * (np.abs(u) + scale / l1))
    # in-place sweep is rejected (Jacobi reads u everywhere)
    assert L.amgt_bsr_jacobi(0, ctypes.byref(G.s), inv.data_ptr(), 0.8, fd.data_ptr(), ud.data_ptr(),
                             ud.data_ptr(), st) == 1


def _hier(orc, dims):
    A = orc.laplacian(*dims) if dims[2] > 0 else None
    return A, orc.geometric_hierarchy(*dims)


def _gpu_solver(amgt, A, Ps, **kw):
    from amgt_b200.amg import AmgSolver, default_params

    return AmgSolver(to_dev(A), [to_dev(P) for P in Ps], default_params(**kw))


@pytest.mark.parametrize("dims", [(64, 64, 1), (128, 128, 1), (24, 20, 16), (48, 48, 48)])
@pytest.mark.parametrize("use_graph", [1, 0])
def test_amg_pcg_fp64_matches_oracle(amgt, orc, dims, use_graph):
    amgt.set_level_policy([0])  # plain fp64
    A = orc.laplacian(*dims)
    Ps = orc.geometric_hierarchy(*dims)
    xs = orc.rand_uniform(0, A.n)
    b = A.to_scipy() @ xs
    xo, it_o, rel_o, hist_o = orc.Amg(A, Ps).solve(b)
    S = _gpu_solver(amgt, A, Ps, use_graph=use_graph)
    assert S.num_levels() == len(Ps) + 1
    x, it, rel = S.solve(torch.from_numpy(b).cuda())
    assert it == it_o
    np.testing.assert_allclose(S.history(), hist_o, rtol=1e-6)
    assert rel <= 1e-8
    xg = x.cpu().numpy()
    assert np.linalg.norm(xg - xo) <= 1e-9 * np.linalg.norm(xo)
    # verified in fp64 on the CPU
    r = b - A.to_scipy() @ xg
    assert np.linalg.norm(r) <= 1.0000001e-8 * np.linalg.norm(b)


def test_amg_levels_match_oracle_galerkin(amgt, orc):
    amgt.set_level_policy([0])
    dims = (20, 18, 16)
    A = orc.laplacian(*dims)
    Ps = orc.geometric_hierarchy(*dims)
    S = _gpu_solver(amgt, A, Ps)
    want = orc.Amg(A, Ps).levels()
    for l, (n, nb) in enumerate(want):
        info = S.level(l)
        assert (info["rows"], info["blocks"]) == (n, nb)


@pytest.mark.parametrize("max_iter", [100, 4])
def test_amg_graph_and_direct_launches_agree_bit_for_bit(amgt, orc, max_iter):
    """The graph path (the whole PCG loop as one launch: a conditional while
    node whose body ends with the convergence test) and direct launches with
    a host test per iteration give the same x, iteration count and residual
    history, also when max_iter stops the loop and on a second solve that
    reuses the built graph."""
    amgt.set_level_policy([0])
    try:
        dims = (40, 36, 32)
        A = orc.laplacian(*dims)
        Ps = orc.geometric_hierarchy(*dims)
        S1 = _gpu_solver(amgt, A, Ps, use_graph=1, max_iter=max_iter)
        S2 = _gpu_solver(amgt, A, Ps, use_graph=0, max_iter=max_iter)
        x1 = torch.zeros(A.n, dtype=torch.float64, device="cuda")  # the same x buffer: the graph is reused
        x2 = torch.zeros_like(x1)
        for seed in (4, 5):
            b = torch.from_numpy(A.to_scipy() @ orc.rand_uniform(seed, A.n)).cuda()
            x1.zero_()
            x2.zero_()
            _, it1, r1 = S1.solve(b, x1)
            _, it2, r2 = S2.solve(b, x2)
            assert it1 == it2 and r1 == r2
            if max_iter == 4:
                assert it1 == 4 and r1 > 1e-8
            else:
                assert it1 < max_iter and r1 <= 1e-8
            assert torch.equal(x1, x2)
            assert np.array_equal(S1.history(), S2.history())
    finally:
        amgt.set_level_policy([])


def test_amg_setup_orders_inputs_still_being_copied(amgt, orc):
    """Setup runs part of its work on a second stream; inputs whose copies
    from pinned host memory are still in flight on the caller's stream must
    be complete before that stream reads them (same x, bit for bit, as with
    blocking copies)."""
    from amgt_b200.amg import AmgSolver, default_params

    amgt.set_level_policy([0])
    try:
        dims = (40, 36, 32)
        A = orc.laplacian(*dims)
        Ps = orc.geometric_hierarchy(*dims)
        b = orc.rand_uniform(4, A.n)

        def pinned(M):
            return (M.m, M.n) + tuple(torch.from_numpy(v).pin_memory() for v in (M.ia, M.ja, M.a))

        def nonblocking(M):
            return M[:2] + tuple(t.cuda(non_blocking=True) for t in M[2:])

        hA, hPs = pinned(A), [pinned(P) for P in Ps]
        torch.cuda.synchronize()
        S = AmgSolver(nonblocking(hA), [nonblocking(P) for P in hPs], default_params())
        x1, it1, _ = S.solve(torch.from_numpy(b).pin_memory().cuda(non_blocking=True))
        x0, it0, _ = _gpu_solver(amgt, A, Ps).solve(torch.from_numpy(b).cuda())
        assert it1 == it0
        assert torch.equal(x1.view(torch.int64), x0.view(torch.int64))
    finally:
        amgt.set_level_policy([])


@pytest.mark.parametrize("problem", ["laplacian", "varcoef27"])
def test_amg_exact_storage_changes_no_bit(amgt, orc, problem):
    """fp64 AMG-PCG with the operators read from exact fp16 / fp32 shadows
    (exact_storage = 1, the default) returns the same x, bit for bit, and
    the same iteration count as with 8-byte values: on the 7-point operator
    (fp16-exact levels) and on a variable-coefficient one whose values no
    narrow format holds (every exactness check, fused or not, must say so)."""
    amgt.set_level_policy([0])
    try:
        dims = (40, 36, 32)
        A = orc.laplacian(*dims) if problem == "laplacian" else orc.varcoef27(*dims, seed=3)
        Ps = orc.geometric_hierarchy(*dims)
        b = torch.from_numpy(A.to_scipy() @ orc.rand_uniform(4, A.n)).cuda()
        x1, it1, r1 = _gpu_solver(amgt, A, Ps, exact_storage=1).solve(b)
        x0, it0, r0 = _gpu_solver(amgt, A, Ps, exact_storage=0).solve(b)
        assert it1 == it0 and r1 == r0
        assert torch.equal(x1.view(torch.int64), x0.view(torch.int64))
    finally:
        amgt.set_level_policy([])


def _reverse_some_rows(orc, M, count):
    """M with the entries of its first `count` rows of two or more entries
    in reverse (unsorted) order."""
    lens = np.diff(M.ia)
    rows = np.nonzero(lens >= 2)[0][:count]
    ja, a = M.ja.copy(), M.a.copy()
    for r in rows:
        lo, hi = M.ia[r], M.ia[r + 1]
        ja[lo:hi] = ja[lo:hi][::-1]
        a[lo:hi] = a[lo:hi][::-1]
    return orc.CSR(M.m, M.n, M.ia, ja, a)


@pytest.mark.parametrize("exact", [1, 0])
def test_amg_setup_work_fused_into_conversion_changes_no_bit(amgt, orc, exact):
    """When every block row of A (of P) takes the conversion's sorted path,
    its fill pass also writes level 0's l1 norms and, with exact storage,
    the fp16 shadow and exactness bits; with a few rows given in reverse
    order the separate passes run instead.  Both setups give the same x,
    iteration count and residual, bit for bit."""
    amgt.set_level_policy([0])
    try:
        dims = (40, 36, 32)
        A = orc.laplacian(*dims)
        Ps = orc.geometric_hierarchy(*dims)
        Ar = _reverse_some_rows(orc, A, 5)
        Psr = [_reverse_some_rows(orc, P, 3) for P in Ps]
        b = torch.from_numpy(A.to_scipy() @ orc.rand_uniform(6, A.n)).cuda()
        x1, it1, r1 = _gpu_solver(amgt, A, Ps, exact_storage=exact).solve(b)
        x2, it2, r2 = _gpu_solver(amgt, Ar, Psr, exact_storage=exact).solve(b)
        assert it1 == it2 and r1 == r2
        assert torch.equal(x1.view(torch.int64), x2.view(torch.int64))
    finally:
        amgt.set_level_policy([])


@pytest.mark.parametrize("policy,flexible", [([0, 1], 0), ([0, 1, 1, 2], 1), ([0, 1, 1, 3], 1)])
def test_amg_mixed_precision_converges_fp64_verified(amgt, orc, policy, flexible):
    amgt.set_level_policy(policy)
    try:
        A = orc.varcoef27(32, 30, 28, seed=1)
        Ps = orc.geometric_hierarchy(32, 30, 28)
        xs = orc.rand_uniform(0, A.n)
        b = A.to_scipy() @ xs
        xo, it_o, _, _ = orc.Amg(A, Ps).solve(b)
        S = _gpu_solver(amgt, A, Ps, flexible=flexible, smooth_prec0=1)
        x, it, rel = S.solve(torch.from_numpy(b).cuda())
        xg = x.cpu().numpy()
        r = b - A.to_scipy() @ xg
        assert np.linalg.norm(r) <= 1.0000001e-8 * np.linalg.norm(b)
        assert it <= it_o + 3
        err = np.linalg.norm(xg - xo) / np.linalg.norm(xo)
        assert err < 1e-6
    finally:
        amgt.set_level_policy([])


def test_amg_solve_reuses_setup_and_initial_guess(amgt, orc):
    amgt.set_level_policy([0])
    A = orc.laplacian(30, 30, 1)
    Ps = orc.geometric_hierarchy(30, 30, 1)
    S = _gpu_solver(amgt, A, Ps)
    b = torch.from_numpy(A.to_scipy() @ orc.rand_uniform(8, A.n)).cuda()
    x, it, rel = S.solve(b)
    # starting from the solution: zero iterations
    x2, it2, rel2 = S.solve(b, x.clone())
    assert it2 == 0 and rel2 <= 1e-8
    # second right-hand side through the same hierarchy
    b3 = torch.from_numpy(A.to_scipy() @ orc.rand_uniform(9, A.n)).cuda()
    _, it3, rel3 = S.solve(b3)
    assert rel3 <= 1e-8 and abs(it3 - it) <= 2


def test_amg_single_level_dense_inverse_exact(amgt, orc):
    """One level: the coarsest (only) operator is inverted exactly (Cholesky
    when it exists, else Gauss-Jordan with partial pivoting), so PCG with
    that preconditioner converges in one iteration, also for a
    non-symmetric matrix with a zero first pivot."""
    import scipy.sparse as sp

    rng = np.random.default_rng(7)
    n = 40
    M = rng.standard_normal((n, n))
    M[0, 0] = 0.0  # first pivot would be zero without row exchanges
    M += np.diag(np.where(np.arange(n) == 0, 0.0, n))
    S = sp.csr_matrix(M)
    A = orc.CSR(n, n, S.indptr.astype(np.int32), S.indices.astype(np.int32), S.data.copy())
    b = rng.standard_normal(n)
    amgt.set_level_policy([0])
    try:
        x, it, rel = _gpu_solver(amgt, A, []).solve(torch.from_numpy(b).cuda())
        assert it == 1 and rel <= 1e-12
        np.testing.assert_allclose(x.cpu().numpy(), np.linalg.solve(M, b), rtol=1e-10, atol=1e-12)
    finally:
        amgt.set_level_policy([])


def test_amg_singular_coarsest_is_reported(amgt, orc):
    """A zero row makes the coarsest operator singular: setup returns
    AMGT_ERR_INVALID (the elimination finds a zero pivot)."""
    from amgt_b200._lib import AmgtError

    A = orc.laplacian(4, 4, 2)
    a = A.a.copy()
    a[A.ia[5]:A.ia[6]] = 0.0
    amgt.set_level_policy([0])
    try:
        with pytest.raises(AmgtError) as ei:
            _gpu_solver(amgt, orc.CSR(A.m, A.n, A.ia, A.ja, a), [])
        assert ei.value.status == 1
    finally:
        amgt.set_level_policy([])


@pytest.mark.parametrize("kind", ["7pt_40", "varcoef27_28"])
@pytest.mark.parametrize("mixed", [0, 1])
def test_fgmres_ir_converges_and_matches_fp64_oracle(amgt, orc, kind, mixed):
    """FGMRES(30) with iterative refinement: the fp64 residual reaches 1e-8
    (checked again by the oracle in fp64), and x agrees with the oracle's
    fp64 AMG-PCG solution of the same system to 1e-6 relative (both stop at
    a relative residual of 1e-8).  mixed: levels 1-2 fp32, >= 3 fp16, level
    0 inside the inner solve in fp32 (exact fp16 storage where it holds)."""
    from amgt_b200 import _lib

    dims = (40, 36, 32) if kind == "7pt_40" else (28, 26, 24)
    A = orc.laplacian(*dims) if kind == "7pt_40" else orc.varcoef27(*dims, seed=1)
    Ps = orc.geometric_hierarchy(*dims)
    b = orc.rand_uniform(0, A.n)
    xo, it_o, _, _ = orc.Amg(A, Ps).solve(b)
    amgt.set_level_policy([0, 1, 1, 2] if mixed else [0])
    try:
        kw = dict(solver=_lib.SOLVER_FGMRES_IR, inner_prec0=1 if mixed else 0, smooth_prec0=1 if mixed else 0,
                  galerkin_by_level=mixed)
        S = _gpu_solver(amgt, A, Ps, **kw)
        x, it, rel = S.solve(torch.from_numpy(b).cuda())
        hist = S.history()
        S.free()
    finally:
        amgt.set_level_policy([])
    assert rel <= 1e-8 and 0 < it <= 40
    assert hist[-1] == pytest.approx(rel)
    xg = x.cpu().numpy()
    assert np.linalg.norm(b - A.to_scipy() @ xg) <= 1.0000001e-8 * np.linalg.norm(b)
    assert np.linalg.norm(xg - xo) <= 1e-6 * np.linalg.norm(xo)


def test_fgmres_ir_graph_and_direct_launches_agree_bit_for_bit(amgt, orc):
    from amgt_b200 import _lib

    dims = (24, 22, 20)
    A = orc.varcoef27(*dims, seed=2)
    Ps = orc.geometric_hierarchy(*dims)
    b = torch.from_numpy(orc.rand_uniform(3, A.n)).cuda()
    amgt.set_level_policy([0, 1, 2])
    try:
        out = []
        for g in (1, 0):
            S = _gpu_solver(amgt, A, Ps, solver=_lib.SOLVER_FGMRES_IR, use_graph=g, inner_prec0=1)
            for _ in range(2):  # a second solve reuses the built graph
                x, it, rel = S.solve(b)
                out.append((x.clone(), it, rel, S.history()))
            S.free()
    finally:
        amgt.set_level_policy([])
    for x, it, rel, h in out[1:]:
        assert torch.equal(x, out[0][0]) and it == out[0][1] and rel == out[0][2] and h == out[0][3]


def test_fgmres_ir_stops_at_max_iter(amgt, orc):
    from amgt_b200 import _lib

    dims = (32, 32, 32)
    A = orc.laplacian(*dims)
    Ps = orc.geometric_hierarchy(*dims)
    b = torch.from_numpy(orc.rand_uniform(0, A.n)).cuda()
    S = _gpu_solver(amgt, A, Ps, solver=_lib.SOLVER_FGMRES_IR, max_iter=3, inner_tol=1e-12)
    x, it, rel = S.solve(b)
    S.free()
    assert it == 3 and rel > 1e-8
