"""GPU parity of the bitmap-packed mBSR values (amgt_pbsr): packing is
exact (the set bits' values in bitmap order, rounded once to the packed
precision), and SpMV / residual / l1-Jacobi on it match the oracle with the
same bounds as the 16-value kernels, and the 16-value kernels themselves in
fp64."""
import numpy as np
import pytest
import torch

from gpu_util import random_csr, to_dev

pytestmark = pytest.mark.gpu

TOL = {0: 1e-12, 1: 1e-5, 2: 1e-5, 3: 1e-5}


def _mats(orc):
    return {"7pt": orc.laplacian(30, 26, 22), "varcoef27": orc.varcoef27(17, 15, 13, seed=2),
            "ragged": random_csr(orc, 1001, 1234, 20, seed=3), "interp": orc.interp(21, 17, 13)[0],
            # block rows of more values than a segment stages at once (512):
            # the chunk-by-chunk staging
            "long": random_csr(orc, 203, 6000, 40, seed=4, dense_rows={5: 1500, 6: 900, 77: 2500})}


@pytest.fixture(scope="module")
def mats(orc):
    return _mats(orc)


@pytest.mark.parametrize("prec", [0, 1, 2, 3])
def test_pack_values_exact(amgt, orc, mats, prec):
    A = mats["varcoef27"]
    R = orc.csr2bsr(A)
    G = amgt.Bsr.from_csr(*to_dev(A))
    Pk = G.pack(prec)
    assert Pk.s.nnz == A.nnz and Pk.s.blc_num == R.nblk
    from amgt_b200.mbsr import view

    rvoff = view(Pk.s.rowVoff, R.brow + 1, torch.int32).cpu().numpy()
    voff = np.concatenate([[0], np.cumsum([bin(int(m)).count("1") for m in R.bmap])])
    np.testing.assert_array_equal(rvoff, voff[R.bptr])
    mask = ((R.bmap[:, None].astype(np.int64) >> np.arange(16)) & 1).astype(bool)
    want = R.bval.reshape(-1, 16)[mask]  # row-major blocks, set bits in bit order
    n = A.nnz
    if prec == 0:
        got = view(Pk.s.val, n, torch.float64).cpu().numpy()
        np.testing.assert_array_equal(got.view(np.uint64), want.view(np.uint64))
    elif prec == 1:
        got = view(Pk.s.val, n, torch.float32).cpu().numpy()
        np.testing.assert_array_equal(got, want.astype(np.float32))
    else:
        got = view(Pk.s.val, n, torch.int16).cpu().numpy().view(np.uint16)
        np.testing.assert_array_equal(got, orc.make_shadow(prec, want))


@pytest.mark.parametrize("name", ["7pt", "varcoef27", "ragged", "interp", "long"])
@pytest.mark.parametrize("prec", [0, 1, 2, 3])
def test_packed_spmv_matches_oracle(amgt, orc, mats, name, prec):
    A = mats[name]
    R = orc.csr2bsr(A)
    G = amgt.Bsr.from_csr(*to_dev(A))
    Pk = G.pack(prec)
    x = orc.rand_uniform(21, A.n)
    y0 = orc.rand_uniform(22, A.m)
    y = torch.from_numpy(y0).cuda()
    Pk.spmv(torch.from_numpy(x).cuda(), y, alpha=-0.75, beta=1.25)
    want = orc.spmv(R, x, y0, alpha=-0.75, beta=1.25, prec=prec)
    scale = orc.spmv_bound(R, x, y0, alpha=-0.75, beta=1.25)
    assert np.all(np.abs(y.cpu().numpy() - want) <= TOL[prec] * scale + 1e-300)



@pytest.mark.parametrize("name", ["7pt", "varcoef27", "ragged", "interp", "long"])
def test_packed_fp64_spmv_equals_dense_bitwise(amgt, orc, mats, name):
    """fp64 packed values: each lane sums its row of every block as the
    16-value kernel does (same lanes per row, an FMA for every column, zero
    where the bit is clear), so y is the dense SpMV's bit for bit."""
    A = mats[name]
    G = amgt.Bsr.from_csr(*to_dev(A))
    Pk = G.pack(0)
    x = torch.from_numpy(orc.rand_uniform(31, A.n)).cuda()
    y0 = torch.from_numpy(orc.rand_uniform(32, A.m)).cuda()
    yd, yp = y0.clone(), y0.clone()
    G.spmv(x, yd, alpha=-0.75, beta=1.25)
    Pk.spmv(x, yp, alpha=-0.75, beta=1.25)
    assert torch.equal(yd.view(torch.int64), yp.view(torch.int64))


def test_packed_residual_and_jacobi(amgt, orc, mats):
    A = mats["varcoef27"]
    R = orc.csr2bsr(A)
    G = amgt.Bsr.from_csr(*to_dev(A))
    Pk = G.pack(0)
    u = orc.rand_uniform(1, A.n)
    f = orc.rand_uniform(2, A.n)
    l1 = np.asarray(abs(A.to_scipy()).sum(axis=1)).ravel()
    ud, fd = torch.from_numpy(u).cuda(), torch.from_numpy(f).cuda()
    r = Pk.residual(fd, ud).cpu().numpy()
    scale = orc.spmv_bound(R, u, f, alpha=-1.0, beta=1.0)
    assert np.all(np.abs(r - (f - orc.spmv(R, u))) <= 1e-12 * scale)
    out = Pk.jacobi(torch.from_numpy(1.0 / l1).cuda(), 0.9, fd, ud).cpu().numpy()
    want = u + 0.9 * (f - orc.spmv(R, u)) / l1
    assert np.all(np.abs(out - want) <= 1e-12 * (np.abs(u) + scale / l1))


def test_amg_packed_and_dense_paths_agree(amgt, orc):
    from amgt_b200.amg import AmgSolver, default_params

    amgt.set_level_policy([0])
    dims = (36, 32, 28)
    A = orc.laplacian(*dims)
    Ps = orc.geometric_hierarchy(*dims)
    b = torch.from_numpy(A.to_scipy() @ orc.rand_uniform(6, A.n)).cuda()
    Sd = AmgSolver(to_dev(A), [to_dev(P) for P in Ps], default_params(packed=0))
    Sp = AmgSolver(to_dev(A), [to_dev(P) for P in Ps], default_params(packed=1))
    xd, itd, _ = Sd.solve(b)
    xp, itp, _ = Sp.solve(b)
    assert itd == itp
    assert float(torch.linalg.vector_norm(xd - xp) / torch.linalg.vector_norm(xd)) < 1e-12
