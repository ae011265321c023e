"""GPU tests of the HYPRE-named mirror layer (amgt_CSRSpGemm /
amgt_CSRMatrixMatvec): level -> precision dispatch, caching, ownership,
trans and multivector handling, error behaviour."""
import numpy as np
import pytest
import torch

from gpu_util import assert_bsr_equal, to_dev

pytestmark = pytest.mark.gpu


def _mk(amgt, A, level=0):
    m, n, ia, ja, a = to_dev(A)
    return amgt.CSRMatrix.create(m, n, ia, ja, a, level=level)


@pytest.mark.parametrize("level,prec", [(0, 0), (1, 1), (2, 2), (5, 2)])
def test_spgemm_hook_precision_by_level(amgt, orc, level, prec):
    amgt.set_level_policy([])  # default get_calculationPrecison table
    A = orc.varcoef27(12, 11, 9, seed=1)
    P, _ = orc.interp(12, 11, 9)
    HA, HP = _mk(amgt, A, level), _mk(amgt, P, level)
    assert HA.bsr_tag == 0
    C = amgt.hypreDevice_CSRSpGemm(HA, HP)
    assert HA.bsr_tag == 1 and HP.bsr_tag == 1
    assert C.bsr_tag == 1 and C.owns_data == 1 and C.level == level
    RC, _ = orc.spgemm(orc.csr2bsr(A), orc.csr2bsr(P), prec=prec)
    Rc = orc.bsr2csr(RC)
    assert C.num_rows == A.m and C.num_cols == P.n and C.num_nonzeros == Rc.nnz
    np.testing.assert_array_equal(C.i.cpu().numpy(), Rc.ia)
    np.testing.assert_array_equal(C.j.cpu().numpy(), Rc.ja)
    np.testing.assert_array_equal(C.data.cpu().numpy().view(np.uint64), Rc.a.view(np.uint64))
    C.destroy()


def test_galerkin_triple_product_through_hooks(amgt, orc):
    """R*(A*P) as hypre_CSRMatrixTripleMultiplyDevice does it
    (csr_matop_device.c:282-292): two hook calls, keepT transpose."""
    amgt.set_level_policy([])
    A = orc.laplacian(20, 16, 12)
    P, _ = orc.interp(20, 16, 12)
    S = P.to_scipy().T.tocsr()
    S.sort_indices()
    R = orc.CSR(S.shape[0], S.shape[1], S.indptr.astype(np.int32), S.indices.astype(np.int32), S.data.copy())
    HA, HP, HR = _mk(amgt, A), _mk(amgt, P), _mk(amgt, R)
    AP = amgt.hypreDevice_CSRSpGemm(HA, HP)
    RAP = amgt.hypreDevice_CSRSpGemm(HR, AP)
    want = (S @ (A.to_scipy() @ P.to_scipy())).tocsr()
    want.sort_indices()
    np.testing.assert_array_equal(RAP.i.cpu().numpy(), want.indptr)
    np.testing.assert_array_equal(RAP.j.cpu().numpy(), want.indices)
    np.testing.assert_allclose(RAP.data.cpu().numpy(), want.data, rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("trans", [0, 1])
def test_matvec_hook_trans(amgt, orc, trans):
    amgt.set_level_policy([])
    P, _ = orc.interp(15, 14, 10)
    H = _mk(amgt, P)
    S = P.to_scipy()
    nin, nout = (P.m, P.n) if trans else (P.n, P.m)
    x = orc.rand_uniform(1, nin)
    y0 = orc.rand_uniform(2, nout)
    y = torch.from_numpy(y0).cuda()
    amgt.hypre_CSRMatrixMatvecCusparseNewAPI(trans, -1.0, H, torch.from_numpy(x).cuda(), 1.0, y)
    want = y0 - ((S.T @ x) if trans else (S @ x))
    np.testing.assert_allclose(y.cpu().numpy(), want, rtol=1e-12, atol=1e-12)


def test_matvec_hook_multivector_and_caching(amgt, orc):
    amgt.set_level_policy([])
    A = orc.varcoef27(13, 12, 10, seed=9)
    H = _mk(amgt, A)
    S = A.to_scipy()
    X = np.stack([orc.rand_uniform(10 + v, A.n) for v in range(6)])
    Y = torch.zeros(6, A.m, dtype=torch.float64, device="cuda")
    amgt.hypre_CSRMatrixMatvecCusparseNewAPI(0, 1.0, H, torch.from_numpy(X).cuda(), 0.0, Y)
    np.testing.assert_allclose(Y.cpu().numpy(), (S @ X.T).T, rtol=1e-12, atol=1e-12)
    # the mBSR form is cached: a second call launches only SpMV kernels
    n0 = amgt.kernel_launch_count()
    x = torch.from_numpy(X[0]).cuda()
    y = torch.zeros(A.m, dtype=torch.float64, device="cuda")
    amgt.hypre_CSRMatrixMatvecCusparseNewAPI(0, 1.0, H, x, 0.0, y)
    assert amgt.kernel_launch_count() - n0 == 1
    assert_bsr_equal(_bsr_wrap(amgt, H), orc.csr2bsr(A))


def _bsr_wrap(amgt, H):
    B = amgt.Bsr()
    B.s = H.bsr  # borrowed view of the cached struct (not owned)
    return B


def test_matvec_hook_rejects_bad_arguments(amgt, orc):
    A = orc.laplacian(8, 8, 1)
    H = _mk(amgt, A)
    x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    y = torch.zeros(A.m, dtype=torch.float64, device="cuda")
    with pytest.raises(amgt.AmgtError) as e:
        amgt.hypre_CSRMatrixMatvecCusparseNewAPI(0, 1.0, H, x, 0.0, y, offset=3)
    assert e.value.status == 1
    with pytest.raises(amgt.AmgtError):
        amgt.hypre_CSRMatrixMatvecCusparseNewAPI(0, 1.0, H, x[:-1].contiguous(), 0.0, y)


def test_mixed_level_matvec_uses_shadow(amgt, orc):
    """Level 2 under the default policy runs the fp16 shadow with fp32
    accumulation; the result matches the oracle's fp16 SpMV."""
    amgt.set_level_policy([])
    A = orc.varcoef27(11, 10, 9, seed=4)
    H = _mk(amgt, A, level=2)
    x = orc.rand_uniform(4, A.n)
    y = torch.zeros(A.m, dtype=torch.float64, device="cuda")
    amgt.hypre_CSRMatrixMatvecCusparseNewAPI(0, 1.0, H, torch.from_numpy(x).cuda(), 0.0, y)
    R = orc.csr2bsr(A)
    want = orc.spmv(R, x, prec=2)
    scale = orc.spmv_bound(R, x, None)
    assert np.all(np.abs(y.cpu().numpy() - want) <= 1e-5 * scale)


def test_kernels_run_sm100_code(amgt):
    """The device code the B200 runs for this library is the sm_100a build
    (cudaFuncGetAttributes binaryVersion 100), queried at run time."""
    import ctypes

    v = ctypes.c_int(0)
    assert amgt.lib().amgt_kernel_arch(ctypes.byref(v)) == 0
    assert v.value == 100
