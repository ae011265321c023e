"""CPU tests of the oracle: pinned against the reference's own known
answers and fixtures (tests/golden/), then cross-checked with scipy."""
import json
import os
from fractions import Fraction

import numpy as np
import pytest
import scipy.sparse as sp

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_generator_matches_hypre_fixture(orc):
    """7-point 10x10x10 Laplacian equals the operator HYPRE's ij wrote
    (TEST_ij/data/poisson_10x10x10_np1/IJ.A.i4f8): same rows, same column
    order (diagonal first), same values."""
    g = np.load(os.path.join(GOLD, "poisson_10x10x10_np1_A.npz"))
    A = orc.laplacian(10, 10, 10)
    rows = np.repeat(np.arange(A.m, dtype=np.int32), np.diff(A.ia))
    assert A.nnz == int(g["header"][5]) == 6400
    np.testing.assert_array_equal(rows, g["rows"])
    np.testing.assert_array_equal(A.ja, g["cols"])
    np.testing.assert_array_equal(A.a, g["vals"])
    # ij's default right-hand side and initial guess (b = 1, x0 = 0)
    assert np.all(g["b"] == 1.0) and np.all(g["x0"] == 0.0)


def _known_answers():
    d = json.load(open(os.path.join(GOLD, "hypre_spgemm_known_answers.json")))
    seen, out = set(), []
    for c in d["cases"]:
        key = (tuple(c["n"]), c["stencil"], c["job"])
        if key in seen:
            continue
        seen.add(key)
        out.append(c)
    return out


def _build(orc, c):
    nx, ny, nz = c["n"]
    return orc.laplacian(nx, ny, nz) if c["stencil"] in ("7pt", "5pt") else orc.box(nx, ny, nz)


SMALL = [c for c in _known_answers() if np.prod(c["n"]) <= 2_097_152]


@pytest.mark.parametrize("case", SMALL, ids=lambda c: f"{c['stencil']}-{'x'.join(map(str, c['n']))}-job{c['job']}")
def test_spgemm_structure_matches_hypre_known_answers(orc, case):
    """Structural nnz of A*A, A^T*A and Diag(A)*A through the mBSR symbolic
    phase equals HYPRE's recorded nnz (benchmark_spgemm.saved.lassen)."""
    A = _build(orc, case)
    B = orc.csr2bsr(A, values=False)
    if case["job"] == 5:
        n = A.m
        D = orc.CSR(n, n, np.arange(n + 1, dtype=np.int32), np.arange(n, dtype=np.int32), np.ones(n))
        nb, nnz = orc.spgemm_count(orc.csr2bsr(D, values=False), B)
    elif case["job"] == 2:
        nb, nnz = orc.spgemm_count(orc.transpose(B), B)
    else:
        nb, nnz = orc.spgemm_count(B, B)
    assert nnz == case["nnz_cpu"] == case["nnz_gpu"]
    assert case["rows"] == A.m


def test_bitmap_product_matches_boolean_matmul(orc):
    rng = np.random.default_rng(0)
    for _ in range(2000):
        a, b = int(rng.integers(0, 1 << 16)), int(rng.integers(0, 1 << 16))
        A = np.array([(a >> i) & 1 for i in range(16)]).reshape(4, 4)
        B = np.array([(b >> i) & 1 for i in range(16)]).reshape(4, 4)
        C = (A @ B) > 0
        want = sum(1 << i for i in range(16) if C.reshape(-1)[i])
        assert orc.bitmatmul(a, b) == want


def _exact_round(d: float, mant: int, ebits: int) -> float:
    """Round-to-nearest-even of d to a binary format, by exact arithmetic."""
    if d == 0 or not np.isfinite(d):
        return d
    bias = (1 << (ebits - 1)) - 1
    emin, emax = 1 - bias, bias
    sign = -1 if d < 0 else 1
    x = Fraction(abs(d))
    e = x.numerator.bit_length() - x.denominator.bit_length()
    while Fraction(2) ** e > x:
        e -= 1
    while Fraction(2) ** (e + 1) <= x:
        e += 1
    e = max(e, emin)
    ulp = Fraction(2) ** (e - mant)
    q, r = divmod(x, ulp)
    if r > ulp / 2 or (r == ulp / 2 and q % 2 == 1):
        q += 1
    v = q * ulp
    maxv = (2 - Fraction(2) ** -mant) * Fraction(2) ** emax
    if v > maxv:
        return sign * float("inf")
    return sign * float(v)


def test_shadow_rounding_is_correctly_rounded(orc):
    rng = np.random.default_rng(1)
    vals = np.concatenate([rng.standard_normal(3000) * 10.0 ** rng.integers(-9, 6, 3000),
                           [65504.0, 65519.99, 65520.0, 6.0e-8, 2.0 ** -25, 3.0 * 2.0 ** -26, 1e-40, -0.0]])
    half = orc.make_shadow(orc.HALF, vals)
    np.testing.assert_array_equal(half, vals.astype(np.float16).view(np.uint16))
    bf = orc.make_shadow(orc.BF16, vals)
    want = np.array([_exact_round(float(v), 7, 8) for v in vals])
    got = (bf.astype(np.uint32) << 16).view(np.float32).astype(np.float64)
    np.testing.assert_array_equal(got, want)


def test_csr2bsr_roundtrip_and_layout(orc):
    A = orc.varcoef27(9, 7, 5, seed=3)
    B = orc.csr2bsr(A)
    assert B.nblk == len(B.bidx)
    # block columns ascend per block row
    for b in range(B.brow):
        seg = B.bidx[B.bptr[b]:B.bptr[b + 1]]
        assert np.all(np.diff(seg) > 0)
    # bits exactly the CSR pattern; values where bits are set, zero elsewhere
    C = orc.bsr2csr(B)
    S = A.to_scipy().tocsr()
    S.sort_indices()
    np.testing.assert_array_equal(C.ia, S.indptr)
    np.testing.assert_array_equal(C.ja, S.indices)
    np.testing.assert_array_equal(C.a, S.data)
    bits = np.unpackbits(B.bmap.view(np.uint8)).sum()
    assert bits == A.nnz
    vals = B.bval.reshape(-1, 16)
    mask = ((B.bmap[:, None].astype(np.int64) >> np.arange(16)) & 1).astype(bool)
    assert np.all(vals[~mask] == 0.0)
    assert abs(B.avg_nnz - A.nnz / B.nblk) < 1e-12
    lens = np.diff(B.bptr)
    assert abs(B.stand - np.sqrt(((lens - lens.mean()) ** 2).mean())) < 1e-9
    assert B.max_row == lens.max()


def test_csr2bsr_ragged_dims_and_empty_rows(orc):
    # n not divisible by 4, an empty row, diagonal-first order, columns past 4*k
    m, n = 11, 13
    rows = {0: [0, 12, 3], 1: [], 2: [2, 0, 5], 5: [5, 4, 6, 9], 10: [10, 1, 12]}
    ia, ja, a = [0], [], []
    for r in range(m):
        cols = rows.get(r, [r % n])
        ja += cols
        a += [float(r * 100 + c + 1) for c in cols]
        ia.append(len(ja))
    A = orc.CSR(m, n, np.array(ia, np.int32), np.array(ja, np.int32), np.array(a))
    B = orc.csr2bsr(A)
    C = orc.bsr2csr(B)
    S = A.to_scipy().tocsr()
    S.sort_indices()
    np.testing.assert_array_equal(C.ia, S.indptr)
    np.testing.assert_array_equal(C.ja, S.indices)
    np.testing.assert_array_equal(C.a, S.data)
    x = np.linspace(-1, 1, n)
    np.testing.assert_allclose(orc.spmv(B, x), S @ x, rtol=1e-14, atol=1e-12)


def test_spmv_oracle_matches_scipy(orc):
    A = orc.varcoef27(12, 10, 9, seed=5)
    B = orc.csr2bsr(A)
    x = orc.rand_uniform(0, A.n)
    y0 = orc.rand_uniform(7, A.m)
    S = A.to_scipy()
    y = orc.spmv(B, x, y0, alpha=-0.5, beta=2.0)
    np.testing.assert_allclose(y, -0.5 * (S @ x) + 2.0 * y0, rtol=1e-13, atol=1e-13)
    # reduced precisions stay within their unit roundoff of the fp64 product
    bound = orc.spmv_bound(B, x, None)
    for prec, u in ((orc.FLOAT, 2.0 ** -24), (orc.HALF, 2.0 ** -11), (orc.BF16, 2.0 ** -8)):
        yl = orc.spmv(B, x, prec=prec)
        assert np.all(np.abs(yl - S @ x) <= 30 * u * bound + 1e-300)


def test_spgemm_oracle_matches_scipy(orc):
    A = orc.varcoef27(10, 9, 8, seed=2)
    P, _ = orc.interp(10, 9, 8)
    BA, BP = orc.csr2bsr(A), orc.csr2bsr(P)
    C, _ = orc.spgemm(BA, BP)
    Cc = orc.bsr2csr(C)
    S = (A.to_scipy() @ P.to_scipy()).tocsr()
    S.sort_indices()
    # structural pattern of A*P (scipy keeps explicit zeros from cancellation)
    np.testing.assert_array_equal(Cc.ia, S.indptr)
    np.testing.assert_array_equal(Cc.ja, S.indices)
    np.testing.assert_allclose(Cc.a, S.data, rtol=1e-12, atol=1e-14)


def test_spgemm_fma_contraction_follows_the_reference_arithmetic(orc):
    """The contracted fp64 product (the reference's `temp += a * b`, which
    nvcc turns into fma) against a hand-written fma chain on a few blocks,
    and against the uncontracted restatement within 1e-12 of |A| |B|.
    The 27-point operator's blocks hold 10 or more entries, the ones the
    reference multiplies with mma.m8n8k4.f64 (csr_spgemm_device.c:1173)."""
    from fractions import Fraction

    def fma(a, b, c):  # a * b + c exactly, rounded once (Fraction -> float rounds to nearest even)
        return float(Fraction(a) * Fraction(b) + Fraction(c))

    A = orc.varcoef27(9, 8, 7, seed=4)
    BA = orc.csr2bsr(A)
    BP = BA  # A * A: random coefficients, so the products round
    assert max(bin(int(m)).count("1") for m in BA.bmap) >= 10
    C1, _ = orc.spgemm(BA, BP)                  # contracted (default)
    C0, _ = orc.spgemm(BA, BP, contract=False)  # separate multiply and add
    np.testing.assert_array_equal(C1.bidx, C0.bidx)
    np.testing.assert_array_equal(C1.bmap, C0.bmap)
    aa = orc.BSR(BA.m, BA.n, BA.bptr, BA.bidx, BA.bmap, np.abs(BA.bval))
    ap = orc.BSR(BP.m, BP.n, BP.bptr, BP.bidx, BP.bmap, np.abs(BP.bval))
    bound, _ = orc.spgemm(aa, ap)
    assert np.all(np.abs(C1.bval - C0.bval) <= 1e-12 * bound.bval)
    assert np.any(C1.bval != C0.bval)  # the contraction is visible in the last bits
    # block row 0 by hand: C(0, J) = sum over A blocks in stored order of
    # the fma-chained 4x4 products
    pos = {int(j): t for t, j in enumerate(C1.bidx[C1.bptr[0]:C1.bptr[1]])}
    acc = np.zeros((len(pos), 16))
    for p in range(BA.bptr[0], BA.bptr[1]):
        k, ma = int(BA.bidx[p]), int(BA.bmap[p])
        a = BA.bval[16 * p:16 * p + 16]
        for q in range(BP.bptr[k], BP.bptr[k + 1]):
            mb = int(BP.bmap[q])
            mc = orc.bitmatmul(ma, mb)
            if not mc:
                continue
            b = BP.bval[16 * q:16 * q + 16]
            t = pos[int(BP.bidx[q])]
            for r in range(4):
                for c in range(4):
                    if not (mc >> (4 * r + c)) & 1:
                        continue
                    s = 0.0
                    for kk in range(4):
                        if (ma >> (4 * r + kk)) & 1 and (mb >> (4 * kk + c)) & 1:
                            s = fma(a[4 * r + kk], b[4 * kk + c], s)
                    acc[t, 4 * r + c] += s
    got = C1.bval[:16 * len(pos)].reshape(-1, 16)
    np.testing.assert_array_equal(got.view(np.uint64), acc.view(np.uint64))


def test_transpose_oracle(orc):
    P, _ = orc.interp(9, 7, 6)
    B = orc.csr2bsr(P)
    T = orc.transpose(B)
    Tc = orc.bsr2csr(T)
    S = P.to_scipy().T.tocsr()
    S.sort_indices()
    np.testing.assert_array_equal(Tc.ia, S.indptr)
    np.testing.assert_array_equal(Tc.ja, S.indices)
    np.testing.assert_array_equal(Tc.a, S.data)


def test_galerkin_product_is_symmetric(orc):
    A = orc.laplacian(16, 12, 10)
    P, _ = orc.interp(16, 12, 10)
    BA, BP = orc.csr2bsr(A), orc.csr2bsr(P)
    AP, _ = orc.spgemm(BA, BP)
    RAP, _ = orc.spgemm(orc.transpose(BP), AP)
    C = orc.bsr2csr(RAP).to_scipy()
    assert abs(C - C.T).max() < 1e-13


def test_oracle_amg_pcg_converges(orc):
    """The oracle's AMG-PCG (Galerkin hierarchy on mBSR, V(1,1) l1-Jacobi)
    reaches 1e-8 on 2D and 3D Poisson with b = A x*, x* uniform seed 0."""
    for dims, max_it in (((64, 64, 1), 16), ((20, 18, 16), 18)):
        A = orc.laplacian(*dims)
        Ps = orc.geometric_hierarchy(*dims)
        xs = orc.rand_uniform(0, A.n)
        b = A.to_scipy() @ xs
        h = orc.Amg(A, Ps)
        x, it, rel, hist = h.solve(b)
        assert rel <= 1e-8 and it <= max_it
        assert np.linalg.norm(b - A.to_scipy() @ x) <= 1.0000001e-8 * np.linalg.norm(b)
        assert hist[0] == pytest.approx(1.0)
        # Galerkin levels equal P^T A P computed by scipy
        n1, nb1 = h.levels()[1]
        C = (Ps[0].to_scipy().T @ A.to_scipy() @ Ps[0].to_scipy()).tocsr()
        assert n1 == C.shape[0]
