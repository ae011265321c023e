"""GPU parity at the sizes of the headline configurations.

C2, 3D 7-point Poisson 128^3 (2,097,152 rows, 14,581,760 nonzeros, the
operator the SpMV half of the metric is quoted on): CSR -> mBSR bit for bit,
fp64 SpMV per row within 1e-12 * (|A| |x|), and the level-0 Galerkin
products A*P and P^T*(A P) bit for bit against the oracle's restatement of
the reference's fp64 arithmetic; the ||C_gpu - C_host||_F / ||C_host||_F
that HYPRE's ij_mm.c:178-191 prints for a device SpGEMM is also computed
(0 when bit-exact).

C4a, 7-point 64^3 with 32 right-hand sides (seeds 0..31): amgt_spmm, per
vector, against the oracle's SpMV: 1e-12 * scale in fp64, 1e-5 * scale
with the fp32 shadow (fp32 accumulation).

C3, 27-point variable-coefficient diffusion 96^3 (log-normal cell
coefficients, seed 1), mixed precision (levels 1-2 fp32, >= 3 fp16): the
solution's residual checked in fp64 by the oracle (<= 1e-8) and its error
against the oracle's fp64 AMG-PCG solution of the same system, with the
bar 1e-6 relative (both solves stop at a relative residual of 1e-8; the
bar leaves room for the operator's conditioning at a 1e3 coefficient
ratio).
"""
import numpy as np
import pytest
import torch

from gpu_util import assert_bsr_equal, to_dev

pytestmark = pytest.mark.gpu


def _abs_bsr(orc, B):
    return orc.BSR(B.m, B.n, B.bptr, B.bidx, B.bmap, np.abs(B.bval))


def test_c2_128cubed_conversion_spmv_galerkin(amgt, orc):
    dims = (128, 128, 128)
    A = orc.laplacian(*dims)
    assert (A.m, A.nnz) == (2097152, 14581760)
    RA = orc.csr2bsr(A)
    GA = amgt.Bsr.from_csr(*to_dev(A))
    assert GA.nblk == RA.nblk == 3620864
    assert_bsr_equal(GA, RA)

    # fp64 SpMV, y = alpha A x + beta y
    x = orc.rand_uniform(0, A.n)
    y0 = orc.rand_uniform(1, A.m)
    y = torch.from_numpy(y0).cuda()
    GA.spmv(torch.from_numpy(x).cuda(), y, alpha=1.5, beta=-0.5)
    want = orc.spmv(RA, x, y0, alpha=1.5, beta=-0.5)
    scale = orc.spmv_bound(RA, x, y0, alpha=1.5, beta=-0.5)
    assert np.all(np.abs(y.cpu().numpy() - want) <= 1e-12 * scale)

    # level-0 Galerkin products
    P, _ = orc.interp(*dims)
    RP = orc.csr2bsr(P)
    RAP, _ = orc.spgemm(RA, RP)
    RR = orc.transpose(RP)
    RC, _ = orc.spgemm(RR, RAP)
    GP = amgt.Bsr.from_csr(*to_dev(P))
    GAP, _ = amgt.spgemm(GA, GP, want_csr=False)
    assert_bsr_equal(GAP, RAP)
    GR = GP.transpose()
    assert_bsr_equal(GR, RR)
    GC, csr = amgt.spgemm(GR, GAP)
    assert_bsr_equal(GC, RC)
    Rc = orc.bsr2csr(RC)
    np.testing.assert_array_equal(csr.ia.cpu().numpy(), Rc.ia)
    np.testing.assert_array_equal(csr.ja.cpu().numpy(), Rc.ja)
    ga = csr.a.cpu().numpy()
    assert np.linalg.norm(ga - Rc.a) / np.linalg.norm(Rc.a) == 0.0  # ij_mm.c's relative error
    # against the uncontracted restatement: within 1e-12 of |R| (|A| |P|)
    RC_nofma, _ = orc.spgemm(RR, orc.spgemm(RA, RP, contract=False)[0], contract=False)
    bound, _ = orc.spgemm(_abs_bsr(orc, RR), orc.spgemm(_abs_bsr(orc, RA), _abs_bsr(orc, RP))[0])
    assert np.all(np.abs(GC.host()["bval"] - RC_nofma.bval) <= 1e-12 * bound.bval)


@pytest.mark.parametrize("prec,tol", [(0, 1e-12), (1, 1e-5)])
def test_c4a_64cubed_32_rhs_spmm(amgt, orc, prec, tol):
    A = orc.laplacian(64, 64, 64)
    RA = orc.csr2bsr(A)
    GA = amgt.Bsr.from_csr(*to_dev(A))
    if prec:
        GA.make_shadow(prec)
    nv = 32
    X = np.stack([orc.rand_uniform(s, A.n) for s in range(nv)])
    Y0 = np.stack([orc.rand_uniform(100 + s, A.m) for s in range(nv)])
    Y = torch.from_numpy(Y0).cuda()
    GA.spmm(torch.from_numpy(X).cuda(), Y, alpha=-1.0, beta=1.0, prec=prec)
    got = Y.cpu().numpy()
    for v in range(nv):
        want = orc.spmv(RA, X[v], Y0[v], alpha=-1.0, beta=1.0)
        scale = orc.spmv_bound(RA, X[v], Y0[v], alpha=-1.0, beta=1.0)
        assert np.all(np.abs(got[v] - want) <= tol * scale), v


def test_c3_mixed_96cubed_error_vs_fp64_oracle(amgt, orc):
    from amgt_b200.amg import AmgSolver, default_params

    dims = (96, 96, 96)
    A = orc.varcoef27(*dims, seed=1)
    Ps = orc.geometric_hierarchy(*dims)
    b = orc.rand_uniform(0, A.n)
    xo, it_o, rel_o, _ = orc.Amg(A, Ps).solve(b)
    assert rel_o <= 1e-8
    amgt.set_level_policy([0, 1, 1, 2])
    try:
        S = AmgSolver(to_dev(A), [to_dev(P) for P in Ps],
                      default_params(flexible=1, smooth_prec0=1, galerkin_by_level=1))
        x, it, rel = S.solve(torch.from_numpy(b).cuda())
        S.free()
    finally:
        amgt.set_level_policy([])
    xg = x.cpu().numpy()
    r = b - A.to_scipy() @ xg
    assert np.linalg.norm(r) <= 1.0000001e-8 * np.linalg.norm(b)
    err = np.linalg.norm(xg - xo) / np.linalg.norm(xo)
    print(f"C3 mixed: {it} iterations (fp64 oracle {it_o}), error vs fp64 oracle x {err:.3e}")
    assert err <= 1e-6
