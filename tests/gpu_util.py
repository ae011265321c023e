"""Helpers shared by the GPU parity tests (test infrastructure)."""
import numpy as np
import torch


def to_dev(A):
    """oracle CSR -> (m, n, ia, ja, a) on cuda:0."""
    return (A.m, A.n, torch.from_numpy(A.ia).cuda(), torch.from_numpy(A.ja).cuda(), torch.from_numpy(A.a).cuda())


def bsr_host(B):
    h = B.host()
    return h["bptr"], h["bidx"], h["bmap"], h["bval"]


def assert_bsr_equal(gpu, orc_bsr, values=True):
    bptr, bidx, bmap, bval = bsr_host(gpu)
    np.testing.assert_array_equal(bptr, orc_bsr.bptr)
    np.testing.assert_array_equal(bidx, orc_bsr.bidx)
    np.testing.assert_array_equal(bmap, orc_bsr.bmap)
    if values:
        # bit for bit
        np.testing.assert_array_equal(bval.view(np.uint64), orc_bsr.bval.view(np.uint64))


def random_csr(orc, m, n, row_len, seed, dense_rows=()):
    """Random CSR with the diagonal (when in range) first, then random
    distinct columns; rows listed in dense_rows get dense_rows[r] entries."""
    rng = np.random.default_rng(seed)
    ia, ja = [0], []
    lens = dict(dense_rows) if isinstance(dense_rows, dict) else {}
    for r in range(m):
        L = lens.get(r, int(rng.integers(0, row_len + 1)))
        L = min(L, n)
        cols = rng.choice(n, size=L, replace=False)
        if r < n and L > 0:
            cols = cols[cols != r][: L - 1]
            cols = np.concatenate([[r], cols])
        ja.extend(int(c) for c in cols)
        ia.append(len(ja))
    ja = np.array(ja, np.int32)
    a = rng.standard_normal(len(ja))
    return orc.CSR(m, n, np.array(ia, np.int32), ja, a)
