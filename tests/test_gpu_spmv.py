"""GPU parity: mBSR SpMV / SpMM through the C ABI against the oracle.

fp64: |y_gpu - y_oracle| <= 1e-12 * (|alpha| sum|a||x| + |beta||y|) per row
(the two sum in different fixed orders).  fp32 / fp16 / bf16: the values are
the same rounded shadows on both sides and both accumulate in fp32, so the
bound is 1e-5 of the same scale (fp32 summation-order differences)."""
import ctypes

import numpy as np
import pytest
import torch

from gpu_util import random_csr, to_dev

pytestmark = pytest.mark.gpu

TOL = {0: 1e-12, 1: 1e-5, 2: 1e-5, 3: 1e-5}


def _mats(orc):
    return {
        "7pt_24x20x16": orc.laplacian(24, 20, 16),
        "7pt_23x19x15": orc.laplacian(23, 19, 15),  # n % 4 != 0: scalar x loads, 2-byte 4-lane run
        "varcoef27_17x13x11": orc.varcoef27(17, 13, 11, seed=6),
        "ragged_rect": random_csr(orc, 1001, 1234, 20, seed=3),  # n % 4 != 0
        "long_rows": random_csr(orc, 400, 40000, 6, seed=4, dense_rows={8: 3000, 9: 2000, 200: 1500}),
        "interp_T": None,
    }


@pytest.fixture(scope="module")
def mats(orc):
    d = _mats(orc)
    P, _ = orc.interp(21, 17, 13)
    S = P.to_scipy().T.tocsr()
    S.sort_indices()
    d["interp_T"] = orc.CSR(S.shape[0], S.shape[1], S.indptr.astype(np.int32), S.indices.astype(np.int32),
                            S.data.copy())
    return d


def _check(orc, R, x, y0, alpha, beta, prec, got):
    want = orc.spmv(R, x, y0, alpha=alpha, beta=beta, prec=prec)
    scale = orc.spmv_bound(R, x, y0 if beta != 0 else None, alpha=alpha, beta=beta)
    err = np.abs(got - want)
    assert np.all(err <= TOL[prec] * scale + 1e-300), f"max err/scale {np.max(err / (scale + 1e-300))}"


@pytest.mark.parametrize("name", ["7pt_24x20x16", "7pt_23x19x15", "varcoef27_17x13x11", "ragged_rect", "long_rows",
                                  "interp_T"])
@pytest.mark.parametrize("prec", [0, 1, 2, 3])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-0.7, 1.0), (2.5, -0.3)])
def test_spmv_matches_oracle(amgt, orc, mats, name, prec, alpha, beta):
    A = mats[name]
    R = orc.csr2bsr(A)
    G = amgt.Bsr.from_csr(*to_dev(A))
    if prec:
        G.make_shadow(prec)
    x = orc.rand_uniform(11, A.n)
    y0 = orc.rand_uniform(12, A.m)
    y = torch.from_numpy(y0).cuda()
    if beta == 0.0:
        y.fill_(float("nan"))  # beta == 0 must not read y
    G.spmv(torch.from_numpy(x).cuda(), y, alpha=alpha, beta=beta, prec=prec)
    _check(orc, R, x, y0, alpha, beta, prec, y.cpu().numpy())


def test_spmv_segmented_long_rows(amgt, orc, mats):
    """Rows longer than 256 blocks with a segment table take the two-pass
    segmented kernel; results are deterministic run to run."""
    A = mats["long_rows"]
    R = orc.csr2bsr(A)
    assert R.max_row > 256
    G = amgt.Bsr.from_csr(*to_dev(A))
    G.balance()
    x = orc.rand_uniform(3, A.n)
    y0 = orc.rand_uniform(4, A.m)
    outs = []
    for _ in range(3):
        y = torch.from_numpy(y0).cuda()
        G.spmv(torch.from_numpy(x).cuda(), y, alpha=1.5, beta=0.5)
        outs.append(y.cpu().numpy())
    _check(orc, R, x, y0, 1.5, 0.5, 0, outs[0])
    assert all(np.array_equal(outs[0], o) for o in outs[1:])


def test_spmv_misaligned_x(amgt, orc, mats):
    """x starting off a 16-byte boundary takes the scalar-load path."""
    A = mats["varcoef27_17x13x11"]
    R = orc.csr2bsr(A)
    G = amgt.Bsr.from_csr(*to_dev(A))
    x = orc.rand_uniform(5, A.n)
    buf = torch.zeros(A.n + 1, dtype=torch.float64, device="cuda")
    buf[1:] = torch.from_numpy(x).cuda()
    xs = buf[1:]
    assert xs.data_ptr() % 16 != 0
    y = G.spmv(xs)
    _check(orc, R, x, np.zeros(A.m), 1.0, 0.0, 0, y.cpu().numpy())


def test_spmv_deterministic(amgt, orc, mats):
    A = mats["varcoef27_17x13x11"]
    G = amgt.Bsr.from_csr(*to_dev(A))
    x = torch.from_numpy(orc.rand_uniform(9, A.n)).cuda()
    ys = [G.spmv(x).cpu().numpy() for _ in range(4)]
    assert all(np.array_equal(ys[0], y) for y in ys[1:])


@pytest.mark.parametrize("nvec", [1, 3, 5, 8, 11])
@pytest.mark.parametrize("prec", [0, 1])
def test_spmm_matches_per_vector_oracle(amgt, orc, mats, nvec, prec):
    A = mats["varcoef27_17x13x11"]
    R = orc.csr2bsr(A)
    G = amgt.Bsr.from_csr(*to_dev(A))
    if prec:
        G.make_shadow(prec)
    X = np.stack([orc.rand_uniform(100 + v, A.n) for v in range(nvec)])
    Y0 = np.stack([orc.rand_uniform(200 + v, A.m) for v in range(nvec)])
    Y = torch.from_numpy(Y0).cuda()
    G.spmm(torch.from_numpy(X).cuda(), Y, alpha=-1.0, beta=1.0, prec=prec)
    Yg = Y.cpu().numpy()
    for v in range(nvec):
        _check(orc, R, X[v], Y0[v], -1.0, 1.0, prec, Yg[v])


def test_spmv_empty_matrix_scales_y(amgt, orc):
    A = orc.CSR(10, 7, np.zeros(11, np.int32), np.zeros(0, np.int32), np.zeros(0))
    G = amgt.Bsr.from_csr(*to_dev(A))
    y = torch.arange(10, dtype=torch.float64, device="cuda")
    G.spmv(torch.ones(7, dtype=torch.float64, device="cuda"), y, alpha=1.0, beta=3.0)
    np.testing.assert_array_equal(y.cpu().numpy(), 3.0 * np.arange(10))


@pytest.mark.parametrize("name,want", [("7pt_24x20x16", 2), ("7pt_23x19x15", 2), ("interp_T", 2),
                                       ("scaled_7pt", 1), ("varcoef27_17x13x11", 0)])
def test_exact_storage_is_bit_identical(amgt, orc, mats, name, want):
    """amgt_bsr_make_exact picks the narrowest shadow that holds every value
    exactly (fp16: 7-point and interpolation weights; fp32: a 7-point
    operator scaled by 1 + 2^-12; none: variable coefficients), and fp64
    products that read it give the fp64 results bit for bit."""
    from amgt_b200 import _lib as L

    if name == "scaled_7pt":
        A = mats["7pt_24x20x16"]
        A = orc.CSR(A.m, A.n, A.ia, A.ja, A.a * (1.0 + 2.0 ** -12))
    else:
        A = mats[name]
    ref = amgt.Bsr.from_csr(*to_dev(A))
    G = amgt.Bsr.from_csr(*to_dev(A))
    assert G.make_exact() == want
    x = torch.from_numpy(orc.rand_uniform(21, A.n)).cuda()
    y0 = torch.from_numpy(orc.rand_uniform(22, A.m)).cuda()
    for alpha, beta in ((1.0, 0.0), (-0.7, 1.0)):
        y_ref, y = y0.clone(), y0.clone()
        ref.spmv(x, y_ref, alpha=alpha, beta=beta)
        G.spmv(x, y, alpha=alpha, beta=beta)
        assert torch.equal(y.view(torch.int64), y_ref.view(torch.int64))
    if A.m == A.n:  # fused residual r = f - A u
        s = torch.cuda.current_stream().cuda_stream
        r_ref, r = torch.empty_like(y0), torch.empty_like(y0)
        assert L.lib().amgt_bsr_residual(0, ctypes.byref(ref.s), y0.data_ptr(), x.data_ptr(), r_ref.data_ptr(), s) == 0
        assert L.lib().amgt_bsr_residual(0, ctypes.byref(G.s), y0.data_ptr(), x.data_ptr(), r.data_ptr(), s) == 0
        assert torch.equal(r.view(torch.int64), r_ref.view(torch.int64))
