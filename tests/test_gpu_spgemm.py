"""GPU parity: mBSR SpGEMM through the C ABI.

C's block pattern and bitmaps equal the oracle bit for bit; values too, in
every precision: fp64 with the reference's arithmetic (each 4x4 product
entry a k-ordered fused multiply-add chain, products added in A block
order), fp32 / fp16 / bf16 with separate fp32 multiply and add in the same
order; the fused CSR output equals the oracle's mBSR -> CSR.  The
structural nnz of A*A on HYPRE's generators equals the reference's recorded
known answers."""
import json
import os

import numpy as np
import pytest
import torch

from gpu_util import assert_bsr_equal, bsr_host, to_dev

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _pair(orc, kind):
    if kind == "AP_7pt":
        A = orc.laplacian(22, 18, 14)
        P, _ = orc.interp(22, 18, 14)
        return A, P
    if kind == "AP_varcoef27":
        A = orc.varcoef27(19, 15, 13, seed=2)
        P, _ = orc.interp(19, 15, 13)
        return A, P
    if kind == "RAP_varcoef27":
        A = orc.varcoef27(15, 13, 11, seed=3)
        P, _ = orc.interp(15, 13, 11)
        AP = orc.bsr2csr(orc.spgemm(orc.csr2bsr(A), orc.csr2bsr(P))[0])
        S = P.to_scipy().T.tocsr()
        S.sort_indices()
        R = orc.CSR(S.shape[0], S.shape[1], S.indptr.astype(np.int32), S.indices.astype(np.int32), S.data.copy())
        return R, AP
    if kind == "AA_varcoef27":
        # random coefficients on both sides: the fp64 products round, so
        # the fused multiply-add chain is visible in the last bits
        A = orc.varcoef27(14, 12, 11, seed=5)
        return A, A
    if kind == "AA_5pt":
        A = orc.laplacian(70, 66, 1)
        return A, A
    if kind == "AAA_27pt":
        # A * A^2: > 1024 pairs per row (window-sweep symbolic) and > 64 C
        # blocks per row (numeric accumulates in global memory)
        A = orc.box(13, 12, 11)
        A2 = orc.bsr2csr(orc.spgemm(orc.csr2bsr(A), orc.csr2bsr(A))[0])
        return A, A2
    if kind == "AP_7pt_large":
        # enough A block rows (> 64 per SM) for the staged warp-per-row numeric
        A = orc.laplacian(48, 40, 40)
        P, _ = orc.interp(48, 40, 40)
        return A, P
    if kind == "AA_7pt_large":
        # C rows of 17-23 blocks: the staged numeric with 24-block
        # accumulators (random values: every rounding of the order shows)
        T = orc.laplacian(48, 40, 40)
        A = orc.CSR(T.m, T.n, T.ia, T.ja, np.random.default_rng(14).uniform(-1, 1, T.ja.size))
        return A, A
    if kind == "A2A2_9pt":
        # A^2 * A^2 of the 9-point pattern: C rows of 25-27 blocks, the staged
        # numeric with 32-block accumulators
        T = orc.box(200, 200, 1)
        A = orc.CSR(T.m, T.n, T.ia, T.ja, np.random.default_rng(15).uniform(-1, 1, T.ja.size))
        A2 = orc.bsr2csr(orc.spgemm(orc.csr2bsr(A), orc.csr2bsr(A))[0])
        return A2, A2
    if kind == "AAA_7pt_wide":
        # A * A^2 of the 7-point operator: every C row holds 33-64 blocks,
        # enough block rows for the staged numeric, which then accumulates
        # in 64-block shared-memory rows (random values: every rounding of
        # the accumulation order shows)
        T = orc.laplacian(48, 40, 40)
        A = orc.CSR(T.m, T.n, T.ia, T.ja, np.random.default_rng(11).uniform(-1, 1, T.ja.size))
        A2 = orc.bsr2csr(orc.spgemm(orc.csr2bsr(A), orc.csr2bsr(A))[0])
        return A, A2
    if kind == "AA_27pt_wide":
        # A * A of the 27-point pattern: C rows of 50-75 blocks (64-block
        # shared accumulators, the longer rows in global memory)
        T = orc.box(40, 40, 24)
        A = orc.CSR(T.m, T.n, T.ia, T.ja, np.random.default_rng(12).uniform(-1, 1, T.ja.size))
        return A, A
    if kind == "LONG_row_staged":
        # the 7-point operator with its first four rows made long (every
        # second column of the first 4,000): one block row of > 1024 pairs
        # and > 64 C blocks among 19,200 short ones, so the staged numeric
        # takes it (pairs found by searching the row's pattern, values
        # accumulated in global memory)
        T = orc.laplacian(48, 40, 40)
        rng = np.random.default_rng(13)
        ia, ja = T.ia.astype(np.int64), T.ja
        long_cols = np.arange(0, 4000, 2, dtype=np.int32)
        rows = [long_cols] * 4 + [ja[ia[i]:ia[i + 1]] for i in range(4, T.m)]
        nia = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
        nja = np.concatenate(rows).astype(np.int32)
        A = orc.CSR(T.m, T.n, nia, nja, rng.uniform(-1, 1, nja.size))
        B = orc.CSR(T.m, T.n, T.ia, T.ja, rng.uniform(-1, 1, T.ja.size))
        return A, B
    if kind == "A2A3_27pt_long":
        # A^2 * A^3 of the 27-point pattern: rows of 4,000-9,800 pairs into at
        # most 484 C blocks (the gathered numeric's order pass on long rows)
        T = orc.box(16, 14, 13)
        A = orc.CSR(T.m, T.n, T.ia, T.ja, np.random.default_rng(16).uniform(-1, 1, T.ja.size))
        A2 = orc.bsr2csr(orc.spgemm(orc.csr2bsr(A), orc.csr2bsr(A))[0])
        A3 = orc.bsr2csr(orc.spgemm(orc.csr2bsr(A2), orc.csr2bsr(A))[0])
        return A2, A3
    if kind == "WIDE_row":
        # a dense first row: > 1024 C blocks in one row (the gathered numeric's
        # A-block-at-a-time ordering)
        rng = np.random.default_rng(7)
        n = 5000
        rows = [np.arange(n)] + [np.unique(rng.integers(0, n, 5)) for _ in range(15)]
        ia = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
        ja = np.concatenate(rows).astype(np.int32)
        A = orc.CSR(16, n, ia, ja, rng.uniform(-1, 1, ja.size))
        T = orc.laplacian(n, 1, 1)
        B = orc.CSR(T.m, T.n, T.ia, T.ja, rng.uniform(-1, 1, T.ja.size))
        return A, B
    raise KeyError(kind)


KINDS = ["AP_7pt", "AP_varcoef27", "RAP_varcoef27", "AA_varcoef27", "AA_5pt", "AAA_27pt", "AP_7pt_large",
         "AA_7pt_large", "A2A2_9pt", "AAA_7pt_wide", "AA_27pt_wide", "LONG_row_staged", "A2A3_27pt_long", "WIDE_row"]


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("prec", [0, 1, 2, 3])
def test_spgemm_bit_exact(amgt, orc, kind, prec):
    A, B = _pair(orc, kind)
    RA, RB = orc.csr2bsr(A), orc.csr2bsr(B)
    RC, Rsh = orc.spgemm(RA, RB, prec=prec)
    GA, GB = amgt.Bsr.from_csr(*to_dev(A)), amgt.Bsr.from_csr(*to_dev(B))
    GC, csr = amgt.spgemm(GA, GB, prec=prec)
    assert GC.nblk == RC.nblk
    assert_bsr_equal(GC, RC)
    if prec:
        got = GC.shadow(prec).cpu().numpy()
        if prec == 1:
            np.testing.assert_array_equal(got.view(np.uint32), Rsh.view(np.uint32))
        else:
            np.testing.assert_array_equal(got.view(np.uint16), Rsh)
    Rc = orc.bsr2csr(RC)
    np.testing.assert_array_equal(csr.ia.cpu().numpy(), Rc.ia)
    np.testing.assert_array_equal(csr.ja.cpu().numpy(), Rc.ja)
    np.testing.assert_array_equal(csr.a.cpu().numpy().view(np.uint64), Rc.a.view(np.uint64))
    assert GC.s.csr_nnz == Rc.nnz
    lens = np.diff(RC.bptr)
    assert GC.s.max_blc_per_row == lens.max()


@pytest.mark.parametrize("kind", ["AP_7pt", "RAP_varcoef27", "AA_varcoef27", "AAA_27pt", "AP_7pt_large", "WIDE_row"])
@pytest.mark.parametrize("prec", [2, 3])
def test_spgemm_tensor_core_engine(amgt, orc, kind, prec):
    """fp16 / bf16 block products on the tensor cores (mma.m16n8k16, fp32
    accumulation, four C blocks per MMA): the pattern and bitmaps equal the
    oracle's bit for bit; every value is within 1e-5 of (|A||B|) of the
    oracle's sequential fp32 result on the same rounded values (the tensor
    core sums in its own order); the CSR form carries the same values."""
    A, B = _pair(orc, kind)
    RA, RB = orc.csr2bsr(A), orc.csr2bsr(B)
    RC, _ = orc.spgemm(RA, RB, prec=prec)
    absA = orc.CSR(A.m, A.n, A.ia, A.ja, np.abs(A.a))
    absB = orc.CSR(B.m, B.n, B.ia, B.ja, np.abs(B.a))
    bound, _ = orc.spgemm(orc.csr2bsr(absA), orc.csr2bsr(absB), prec=0)
    GA, GB = amgt.Bsr.from_csr(*to_dev(A)), amgt.Bsr.from_csr(*to_dev(B))
    assert amgt.lib().amgt_spgemm_set_engine(2) == 0
    try:
        GC, csr = amgt.spgemm(GA, GB, prec=prec)
    finally:
        amgt.lib().amgt_spgemm_set_engine(0)
    assert_bsr_equal(GC, RC, values=False)
    got = bsr_host(GC)[3]
    tol = 1e-5 * bound.bval + 1e-30
    assert np.all(np.abs(got - RC.bval) <= tol), np.max(np.abs(got - RC.bval) / (bound.bval + 1e-300))
    Rc = orc.bsr2csr(RC)
    np.testing.assert_array_equal(csr.ja.cpu().numpy(), Rc.ja)
    Gc = orc.bsr2csr(orc.BSR(GC.s.row, GC.s.col, *bsr_host(GC)))
    np.testing.assert_array_equal(csr.a.cpu().numpy(), Gc.a)


def test_spgemm_fp64_matches_scipy(amgt, orc):
    A, P = _pair(orc, "AP_varcoef27")
    GC, csr = amgt.spgemm(amgt.Bsr.from_csr(*to_dev(A)), amgt.Bsr.from_csr(*to_dev(P)))
    S = (A.to_scipy() @ P.to_scipy()).tocsr()
    S.sort_indices()
    np.testing.assert_array_equal(csr.ia.cpu().numpy(), S.indptr)
    np.testing.assert_array_equal(csr.ja.cpu().numpy(), S.indices)
    np.testing.assert_allclose(csr.a.cpu().numpy(), S.data, rtol=1e-12, atol=1e-14)


def test_spgemm_empty_operands(amgt, orc):
    E = orc.CSR(12, 10, np.zeros(13, np.int32), np.zeros(0, np.int32), np.zeros(0))
    B = orc.laplacian(10, 1, 1)
    GC, csr = amgt.spgemm(amgt.Bsr.from_csr(*to_dev(E)), amgt.Bsr.from_csr(*to_dev(B)))
    assert GC.nblk == 0 and csr.s.num_nonzeros == 0
    np.testing.assert_array_equal(csr.ia.cpu().numpy(), np.zeros(13))


def _known():
    d = json.load(open(os.path.join(GOLD, "hypre_spgemm_known_answers.json")))
    seen, out = set(), []
    for c in d["cases"]:
        key = (tuple(c["n"]), c["stencil"], c["job"])
        if key not in seen:
            seen.add(key)
            out.append(c)
    return out


@pytest.mark.parametrize("case", _known(), ids=lambda c: f"{c['stencil']}-{'x'.join(map(str, c['n']))}-job{c['job']}")
def test_spgemm_structure_matches_hypre_known_answers(amgt, orc, case):
    """Structural nnz of the product (A*A, A^T*A, Diag(A)*A) through the GPU
    symbolic + numeric path equals HYPRE's recorded nnz, up to the
    256x256x128 27-point case (1.03e9 nonzeros; CSR output skipped)."""
    nx, ny, nz = case["n"]
    A = orc.laplacian(nx, ny, nz) if case["stencil"] in ("7pt", "5pt") else orc.box(nx, ny, nz)
    G = amgt.Bsr.from_csr(*to_dev(A))
    if case["job"] == 5:
        n = A.m
        dev = torch.arange(n + 1, dtype=torch.int32, device="cuda")
        L = amgt.Bsr.from_csr(n, n, dev, dev[:-1].contiguous(), torch.ones(n, dtype=torch.float64, device="cuda"))
        R = G
    elif case["job"] == 2:
        L, R = G.transpose(), G
    else:
        L, R = G, G
    del A
    C, _ = amgt.spgemm(L, R, want_csr=False)
    assert C.s.csr_nnz == case["nnz_cpu"]
    C.free()
    torch.cuda.empty_cache()


def test_two_host_threads_on_one_device(amgt, orc):
    """Two host threads convert and multiply at once, each on its own
    stream: every size read-back goes through that thread's own pinned
    staging, so both results stay bit-exact."""
    import threading

    A = orc.laplacian(24, 20, 16)
    P, _ = orc.interp(24, 20, 16)
    RC, _ = orc.spgemm(orc.csr2bsr(A), orc.csr2bsr(P))
    results, errors = [None, None], []

    def work(i):
        try:
            torch.cuda.set_device(0)
            st = torch.cuda.Stream()
            with torch.cuda.stream(st):
                outs = []
                for _ in range(20):
                    GA = amgt.Bsr.from_csr(*to_dev(A), stream=st)
                    GP = amgt.Bsr.from_csr(*to_dev(P), stream=st)
                    GC, _ = amgt.spgemm(GA, GP, want_csr=False, stream=st)
                    outs.append(GC)
                st.synchronize()
                results[i] = outs
        except Exception as e:  # reported by the main thread
            errors.append(e)

    threads = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for outs in results:
        for GC in outs:
            assert_bsr_equal(GC, RC)
