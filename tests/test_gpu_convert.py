"""GPU parity: CSR -> mBSR, mBSR -> CSR, block transpose and value shadows
through the C ABI, bit for bit against the oracle."""
import numpy as np
import pytest
import torch

from gpu_util import assert_bsr_equal, random_csr, to_dev

pytestmark = pytest.mark.gpu


def _reverse_rows(orc, A, rows):
    """A with the entries of the given rows in reverse (unsorted) order."""
    ja, a = A.ja.copy(), A.a.copy()
    for r in rows:
        lo, hi = A.ia[r], A.ia[r + 1]
        ja[lo:hi] = ja[lo:hi][::-1]
        a[lo:hi] = a[lo:hi][::-1]
    return orc.CSR(A.m, A.n, A.ia, ja, a)


def _with_long_row(orc, A, r, length, seed):
    """A with row r replaced by `length` sorted random columns."""
    rng = np.random.default_rng(seed)
    cols = np.sort(rng.choice(A.n, size=length, replace=False)).astype(np.int32)
    rows_ja = [A.ja[A.ia[i]:A.ia[i + 1]] for i in range(A.m)]
    rows_a = [A.a[A.ia[i]:A.ia[i + 1]] for i in range(A.m)]
    rows_ja[r], rows_a[r] = cols, rng.standard_normal(length)
    ia = np.concatenate([[0], np.cumsum([len(x) for x in rows_ja])]).astype(np.int32)
    return orc.CSR(A.m, A.n, ia, np.concatenate(rows_ja).astype(np.int32), np.concatenate(rows_a))


def _with_rows(orc, A, new_rows, seed):
    """A with the rows in new_rows (row -> sorted columns) replaced."""
    rng = np.random.default_rng(seed)
    rows_ja = [A.ja[A.ia[i]:A.ia[i + 1]] for i in range(A.m)]
    rows_a = [A.a[A.ia[i]:A.ia[i + 1]] for i in range(A.m)]
    for r, cols in new_rows.items():
        rows_ja[r] = np.asarray(cols, np.int32)
        rows_a[r] = rng.standard_normal(len(cols))
    ia = np.concatenate([[0], np.cumsum([len(x) for x in rows_ja])]).astype(np.int32)
    return orc.CSR(A.m, A.n, ia, np.concatenate(rows_ja).astype(np.int32), np.concatenate(rows_a))


def _cases(orc):
    lap = orc.laplacian(16, 16, 16)
    return {
        # sorted rows (one thread per block row) mixed with reversed ones in
        # the same warps (the warp kernel), and a warp whose entries do not
        # fit the shared-memory copy because of one long row
        "sorted_some_reversed": _reverse_rows(orc, lap, [7, 100, 101, 102, 103, 2000, 4095]),
        "sorted_one_long": _with_long_row(orc, lap, 300, 1500, seed=5),
        # sorted block rows of more than 32 entries: 128 entries in 32 block
        # columns (the most the one-thread path takes), and 61 entries in
        # more than 32 block columns (left to the warp kernel mid-merge)
        "sorted_wide_block_rows": _with_rows(
            orc, lap, {**{44 + q: [4 * j + c for j in range(100 + 8 * q, 108 + 8 * q) for c in range(4)]
                          for q in range(4)},
                       40: sorted(np.random.default_rng(7).choice(np.arange(0, 4096, 4), 40, replace=False))},
            seed=8),
        "hypre7pt_10x10x10": orc.laplacian(10, 10, 10),
        "5pt_64x64": orc.laplacian(64, 64, 1),
        "varcoef27_13x11x9": orc.varcoef27(13, 11, 9, seed=4),
        "27pt_20x20x20": orc.box(20, 20, 20),
        "interp_13x11x9": orc.interp(13, 11, 9)[0],
        "ragged_rect": random_csr(orc, 1003, 777, 9, seed=1),
        # block rows of 33..512 entries (shared-memory sort) and > 512 (window sweep,
        # columns spread over > 8192 block columns -> several windows)
        "long_rows": random_csr(orc, 402, 70001, 12, seed=2, dense_rows={5: 40, 17: 300, 100: 700, 101: 2500,
                                                                       399: 9000}),
        "empty": orc.CSR(9, 6, np.zeros(10, np.int32), np.zeros(0, np.int32), np.zeros(0)),
    }


@pytest.fixture(scope="module")
def cases(orc):
    return _cases(orc)


CASE_NAMES = ["hypre7pt_10x10x10", "5pt_64x64", "varcoef27_13x11x9", "27pt_20x20x20", "interp_13x11x9",
              "ragged_rect", "long_rows", "empty", "sorted_some_reversed", "sorted_one_long",
              "sorted_wide_block_rows"]


@pytest.mark.parametrize("name", CASE_NAMES)
def test_csr_to_bsr_bit_exact(amgt, orc, cases, name):
    A = cases[name]
    m, n, ia, ja, a = to_dev(A)
    G = amgt.Bsr.from_csr(m, n, ia, ja, a)
    R = orc.csr2bsr(A)
    assert G.nblk == R.nblk
    assert_bsr_equal(G, R)
    assert G.s.max_blc_per_row == R.max_row
    assert G.s.csr_nnz == A.nnz
    assert abs(G.s.stand - R.stand) <= 1e-9 * max(1.0, R.stand)
    assert abs(G.s.avg_nnz - R.avg_nnz) <= 1e-12 * max(1.0, R.avg_nnz)
    assert G.s.blc_row == (m + 3) // 4 and G.s.blc_col == (n + 3) // 4


@pytest.mark.parametrize("name", ["varcoef27_13x11x9", "ragged_rect", "long_rows", "empty"])
def test_bsr_to_csr_roundtrip(amgt, orc, cases, name):
    A = cases[name]
    G = amgt.Bsr.from_csr(*to_dev(A))
    ia, ja, a = (t.cpu().numpy() for t in G.to_csr())
    R = orc.bsr2csr(orc.csr2bsr(A))
    np.testing.assert_array_equal(ia, R.ia)
    np.testing.assert_array_equal(ja, R.ja)
    np.testing.assert_array_equal(a.view(np.uint64), R.a.view(np.uint64))


@pytest.mark.parametrize("name", ["interp_13x11x9", "ragged_rect", "long_rows"])
def test_block_transpose(amgt, orc, cases, name):
    A = cases[name]
    G = amgt.Bsr.from_csr(*to_dev(A)).transpose()
    R = orc.transpose(orc.csr2bsr(A))
    assert_bsr_equal(G, R)
    lens = np.diff(R.bptr)
    assert G.s.max_blc_per_row == (lens.max() if len(lens) else 0)


@pytest.mark.parametrize("prec", [1, 2, 3])
def test_value_shadows_bit_exact(amgt, orc, prec):
    A = orc.varcoef27(11, 9, 7, seed=8, sigma=6.0, ratio=1e12)  # wide exponent range
    G = amgt.Bsr.from_csr(*to_dev(A))
    G.make_shadow(prec)
    got = G.shadow(prec).cpu().numpy()
    want = orc.make_shadow(prec, orc.csr2bsr(A).bval)
    if prec == 1:
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    else:
        np.testing.assert_array_equal(got.view(np.uint16), want)


def test_balance_segments(amgt, orc, cases):
    A = cases["long_rows"]
    G = amgt.Bsr.from_csr(*to_dev(A))
    G.balance()
    lens = np.diff(orc.csr2bsr(A).bptr)
    segs = (lens + 63) // 64
    assert G.s.warpnum == segs.sum()
    from amgt_b200.mbsr import view

    ptr = view(G.s.rowPtrbyWarp, G.s.blc_row + 1, torch.int32).cpu().numpy()
    idx = view(G.s.rowIdxbyWarp, G.s.warpnum, torch.int32).cpu().numpy()
    np.testing.assert_array_equal(ptr, np.concatenate([[0], np.cumsum(segs)]))
    np.testing.assert_array_equal(idx, np.repeat(np.arange(len(lens)), segs))


@pytest.mark.parametrize("bad", [-1, "n"])
def test_csr_to_bsr_reports_bad_column(amgt, orc, bad):
    """A column index outside [0, n) in an otherwise sorted matrix: the
    kernels check the index before using it and the call returns
    AMGT_ERR_DEVICE; the next conversion on the device is unaffected."""
    from amgt_b200._lib import AmgtError

    A = orc.laplacian(16, 16, 16)
    ja = A.ja.copy()
    ja[A.ia[500] + 1] = A.n if bad == "n" else bad
    with pytest.raises(AmgtError) as ei:
        amgt.Bsr.from_csr(*to_dev(orc.CSR(A.m, A.n, A.ia, ja, A.a)))
    assert ei.value.status == 4  # AMGT_ERR_DEVICE
    G = amgt.Bsr.from_csr(*to_dev(A))
    assert_bsr_equal(G, orc.csr2bsr(A))
