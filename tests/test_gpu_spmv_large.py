"""GPU parity at larger sizes: mBSR SpMV and its fused forms on matrices of
4,000 to 10,000 block rows, every lane-group width of the register kernels
(4 lanes for one block per row, 8 for the 7-point operator, 16 for ~12
blocks per row), n % 4 != 0 with a rectangular shape, and a band of 64 long
block rows among short ones.

Exact narrow storage must give the fp64 kernel's results bit for bit (plain
SpMV, fused residual and l1-Jacobi; fp16 shadows of integer values, fp32
shadows of values scaled by 1 + 2^-12); fp32 / fp16 / bf16 shadows are
checked against the oracle with the bounds of test_gpu_spmv."""
import ctypes

import numpy as np
import pytest
import torch

from gpu_util import random_csr, to_dev

pytestmark = pytest.mark.gpu

TOL = {1: 1e-5, 2: 1e-5, 3: 1e-5}


def _int_valued(orc, A, seed):
    rng = np.random.default_rng(seed)
    return orc.CSR(A.m, A.n, A.ia, A.ja, rng.integers(-8, 9, size=A.a.size).astype(np.float64))


def _diag(orc, m, seed):
    rng = np.random.default_rng(seed)
    ia = np.arange(m + 1, dtype=np.int32)
    return orc.CSR(m, m, ia, np.arange(m, dtype=np.int32), rng.integers(1, 9, size=m).astype(np.float64))


@pytest.fixture(scope="module")
def big(orc):
    band = {r: 12 for r in range(4096, 4096 + 256)}  # 64 block rows of ~48 blocks among rows of ~4
    return {
        "7pt_40x32x32": orc.laplacian(40, 32, 32),  # 6.9 blocks per block row: 8 lanes
        "diag_20000": _diag(orc, 20000, 5),  # 1 block per block row: 4 lanes
        "ragged_rect": _int_valued(orc, random_csr(orc, 20001, 30003, 6, seed=7), 7),  # ~12 blocks: 16 lanes
        "dense_band": _int_valued(orc, random_csr(orc, 24000, 24000, 2, seed=8, dense_rows=band), 8),
    }


NAMES = ["7pt_40x32x32", "diag_20000", "ragged_rect", "dense_band"]


def _bits(t):
    return t.view(torch.int64)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("scale,want", [(1.0, 2), (1.0 + 2.0 ** -12, 1)])
def test_large_exact_storage_bit_identical(amgt, orc, big, name, scale, want):
    from amgt_b200 import _lib as L

    A = big[name]
    A = orc.CSR(A.m, A.n, A.ia, A.ja, A.a * scale)
    ref = amgt.Bsr.from_csr(*to_dev(A))
    G = amgt.Bsr.from_csr(*to_dev(A))
    assert G.s.blc_row >= 4096
    assert G.make_exact() == want
    x = torch.from_numpy(orc.rand_uniform(31, A.n)).cuda()
    y0 = torch.from_numpy(orc.rand_uniform(32, A.m)).cuda()
    for alpha, beta in ((1.0, 0.0), (-0.7, 1.0), (2.5, -0.3)):
        y_ref, y = y0.clone(), y0.clone()
        ref.spmv(x, y_ref, alpha=alpha, beta=beta)
        G.spmv(x, y, alpha=alpha, beta=beta)
        assert torch.equal(_bits(y), _bits(y_ref)), (alpha, beta)
    if A.m != A.n:
        return
    s = torch.cuda.current_stream().cuda_stream
    lib = L.lib()
    r_ref, r = torch.empty_like(y0), torch.empty_like(y0)
    assert lib.amgt_bsr_residual(0, ctypes.byref(ref.s), y0.data_ptr(), x.data_ptr(), r_ref.data_ptr(), s) == 0
    assert lib.amgt_bsr_residual(0, ctypes.byref(G.s), y0.data_ptr(), x.data_ptr(), r.data_ptr(), s) == 0
    assert torch.equal(_bits(r), _bits(r_ref))
    inv_l1 = torch.from_numpy(1.0 / (1.0 + np.abs(orc.rand_uniform(33, A.m)))).cuda()
    u_ref, u = torch.empty_like(y0), torch.empty_like(y0)
    assert lib.amgt_bsr_jacobi(0, ctypes.byref(ref.s), inv_l1.data_ptr(), 0.7, y0.data_ptr(), x.data_ptr(),
                               u_ref.data_ptr(), s) == 0
    assert lib.amgt_bsr_jacobi(0, ctypes.byref(G.s), inv_l1.data_ptr(), 0.7, y0.data_ptr(), x.data_ptr(),
                               u.data_ptr(), s) == 0
    assert torch.equal(_bits(u), _bits(u_ref))


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("prec", [1, 2, 3])
@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (-0.7, 1.0)])
def test_large_shadows_match_oracle(amgt, orc, big, name, prec, alpha, beta):
    A = big[name]
    R = orc.csr2bsr(A)
    G = amgt.Bsr.from_csr(*to_dev(A))
    G.make_shadow(prec)
    x = orc.rand_uniform(34, A.n)
    y0 = orc.rand_uniform(35, A.m)
    y = torch.from_numpy(y0).cuda()
    if beta == 0.0:
        y.fill_(float("nan"))  # beta == 0 must not read y
    G.spmv(torch.from_numpy(x).cuda(), y, alpha=alpha, beta=beta, prec=prec)
    want = orc.spmv(R, x, y0, alpha=alpha, beta=beta, prec=prec)
    scale = orc.spmv_bound(R, x, y0 if beta != 0 else None, alpha=alpha, beta=beta)
    err = np.abs(y.cpu().numpy() - want)
    assert np.all(err <= TOL[prec] * scale + 1e-300), f"max err/scale {np.max(err / (scale + 1e-300))}"


def test_large_repeatable(amgt, orc, big):
    """Two calls give the same bits (fixed row -> lane map, no atomics)."""
    A = big["dense_band"]
    G = amgt.Bsr.from_csr(*to_dev(A))
    G.make_shadow(2)
    x = torch.from_numpy(orc.rand_uniform(36, A.n)).cuda()
    y1 = G.spmv(x, prec=2)
    y2 = G.spmv(x, prec=2)
    assert torch.equal(_bits(y1), _bits(y2))
