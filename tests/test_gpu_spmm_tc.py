"""GPU parity of the row-major multivector SpMM (amgt_spmm_rm) and of the
autotuner.

Tensor-core form (fp32 / fp16 / bf16 values, tf32 mma with a high / low
split): per right-hand side, |y - y_oracle| <= 1e-5 * (|alpha| |A| |x| +
|beta| |y|), y_oracle the oracle's SpMV on the same rounded values with fp32
products (the split carries about 21 of fp32's 24 mantissa bits of x);
CUDA-core form: fp64 at 1e-12, reduced precisions at 1e-5.  Shapes cover
ragged dimensions (n % 4 != 0), empty rows, odd block-row counts (the last
pair has one row) and 1 .. 32 right-hand sides."""
import numpy as np
import pytest
import torch

from gpu_util import random_csr, to_dev

pytestmark = pytest.mark.gpu


def _cases(orc):
    return {
        "7pt_17x13x11": orc.laplacian(17, 13, 11),
        "varcoef27_11x10x9": orc.varcoef27(11, 10, 9, seed=3),
        "ragged": random_csr(orc, 211, 173, 9, seed=8),
    }


@pytest.mark.parametrize("name", ["7pt_17x13x11", "varcoef27_11x10x9", "ragged"])
@pytest.mark.parametrize("prec", [0, 1, 2, 3])
@pytest.mark.parametrize("engine", [1, 2])
@pytest.mark.parametrize("nvec", [1, 7, 16, 32])
def test_spmm_rm_matches_oracle_per_vector(amgt, orc, name, prec, engine, nvec):
    A = _cases(orc)[name]
    R = orc.csr2bsr(A)
    G = amgt.Bsr.from_csr(*to_dev(A))
    if prec:
        G.make_shadow(prec)
    X = np.stack([orc.rand_uniform(10 + v, A.n) for v in range(nvec)], axis=1)
    Y0 = np.stack([orc.rand_uniform(50 + v, A.m) for v in range(nvec)], axis=1)
    Y = torch.from_numpy(np.ascontiguousarray(Y0)).cuda()
    G.spmm_rm(torch.from_numpy(np.ascontiguousarray(X)).cuda(), Y, alpha=-0.75, beta=1.25, prec=prec,
              engine=engine)
    got = Y.cpu().numpy()
    tol = 1e-12 if prec == 0 else 1e-5
    for v in range(nvec):
        want = orc.spmv(R, X[:, v], Y0[:, v], alpha=-0.75, beta=1.25, prec=prec)
        scale = orc.spmv_bound(R, X[:, v], Y0[:, v], alpha=-0.75, beta=1.25)
        assert np.all(np.abs(got[:, v] - want) <= tol * scale + 1e-300), v


def test_spmm_rm_tensor_cores_64cubed_32_rhs_fp64_residual(amgt, orc):
    """C4a: 7-point 64^3, 32 right-hand sides; R = B - A X with the products
    on the tensor cores (fp32 values) and the subtraction in fp64."""
    A = orc.laplacian(64, 64, 64)
    R = orc.csr2bsr(A)
    G = amgt.Bsr.from_csr(*to_dev(A))
    G.make_shadow(1)
    nv = 32
    X = np.ascontiguousarray(np.stack([orc.rand_uniform(v, A.n) for v in range(nv)], axis=1))
    B = np.ascontiguousarray(np.stack([orc.rand_uniform(100 + v, A.m) for v in range(nv)], axis=1))
    Rr = torch.from_numpy(B).cuda()
    G.spmm_rm(torch.from_numpy(X).cuda(), Rr, alpha=-1.0, beta=1.0, prec=1, engine=2)
    got = Rr.cpu().numpy()
    for v in range(nv):
        want = orc.spmv(R, X[:, v], B[:, v], alpha=-1.0, beta=1.0)  # fp64 oracle (the values are exact in fp32)
        scale = orc.spmv_bound(R, X[:, v], B[:, v], alpha=-1.0, beta=1.0)
        assert np.all(np.abs(got[:, v] - want) <= 1e-5 * scale), v


def test_spmm_rm_empty_and_invalid(amgt, orc):
    import ctypes

    E = orc.CSR(10, 7, np.zeros(11, np.int32), np.zeros(0, np.int32), np.zeros(0))
    G = amgt.Bsr.from_csr(*to_dev(E))
    Y = torch.ones(10, 3, dtype=torch.float64, device="cuda")
    G.spmm_rm(torch.ones(7, 3, dtype=torch.float64, device="cuda"), Y, beta=0.5)
    assert torch.all(Y == 0.5)
    L = amgt.lib()
    assert L.amgt_spmm_rm(0, 0, 1.0, ctypes.byref(G.s), 33, Y.data_ptr(), 0.0, Y.data_ptr(), None) == 1
    assert L.amgt_spmm_rm(0, 3, 1.0, ctypes.byref(G.s), 3, Y.data_ptr(), 0.0, Y.data_ptr(), None) == 1


def test_autotuner_picks_a_measured_candidate_and_results_hold(amgt, orc):
    A = orc.laplacian(40, 36, 32)
    R = orc.csr2bsr(A)
    G = amgt.Bsr.from_csr(*to_dev(A))
    G.make_shadow(1)
    # SpMM: engine x warps per CTA
    t = G.autotune(prec=1, nvec=32)
    assert set(t["ms"]) == {4, 8, 14, 18} and t["choice"] in t["ms"]
    assert t["ms"][t["choice"]] == min(t["ms"].values())
    X = np.ascontiguousarray(np.stack([orc.rand_uniform(v, A.n) for v in range(32)], axis=1))
    Y = G.spmm_rm(torch.from_numpy(X).cuda(), prec=1, engine=0).cpu().numpy()
    for v in (0, 31):
        want = orc.spmv(R, X[:, v], prec=1)
        assert np.all(np.abs(Y[:, v] - want) <= 1e-5 * orc.spmv_bound(R, X[:, v], None))
    # SpMV: lanes per block row; fp64 8-byte and exact fp16 storage keep equal sums
    t1 = G.autotune(prec=0, nvec=1)
    assert set(t1["ms"]) == {4, 8, 16, 32} and t1["choice"] in (4, 8, 16, 32)
    x = torch.from_numpy(orc.rand_uniform(7, A.n)).cuda()
    y8 = G.spmv(x).clone()
    want = orc.spmv(R, x.cpu().numpy())
    assert np.all(np.abs(y8.cpu().numpy() - want) <= 1e-12 * orc.spmv_bound(R, x.cpu().numpy(), None))
    assert G.make_exact() == 2
    assert torch.equal(G.spmv(x), y8)
    assert amgt.lib().amgt_autotune_clear() == 0
