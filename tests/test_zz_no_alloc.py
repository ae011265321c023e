"""GPU test of amgt_spmv_segmented_noalloc, the SpMV entry point that
allocates nothing.

It exists for callers that cannot allocate device memory when they run a
matvec: a solver that gave its whole device memory to a pool sized at
set-up, a caller whose allocator may not be called from the thread that
issues the solve, a caller that cannot afford the device-wide
synchronisation cudaMalloc / cudaFree can cause.  Its partial sums live in a
fixed device array of AMGT_NOALLOC_MAX_SEGMENTS * 4 doubles instead.

The test calls it through the C ABI twice in a row and compares each result
with amgt_spmv's (which takes the same segmented path with allocated
scratch), within the SpMV tolerance the other tests use; it checks that the
allocator is never called, and that a segment count beyond the maximum is
rejected.  The file is named to be collected last and builds its own
inputs, so it passes alone in a fresh process and after the other tests.
"""
import ctypes

import numpy as np
import pytest
import torch

from gpu_util import random_csr, to_dev

pytestmark = pytest.mark.gpu

ALLOC_FN = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p)
FREE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p)


def _spmv_noalloc(L, prec, alpha, G, x, beta, y):
    return L.amgt_spmv_segmented_noalloc(prec, alpha, ctypes.byref(G.s), x.data_ptr(), beta, y.data_ptr(),
                                         torch.cuda.current_stream().cuda_stream)


def test_noalloc_spmv_matches_allocating_spmv_twice(amgt, orc):
    L = amgt.lib()
    A = random_csr(orc, 600, 50000, 10, seed=21, dense_rows={3: 5000, 4: 2600, 301: 1200, 599: 900})
    R = orc.csr2bsr(A)
    G = amgt.Bsr.from_csr(*to_dev(A))
    G.balance()
    assert G.s.max_blc_per_row > 256 and 0 < G.s.warpnum <= amgt._lib.NOALLOC_MAX_SEGMENTS
    x = torch.from_numpy(orc.rand_uniform(31, A.n)).cuda()
    y0 = orc.rand_uniform(32, A.m)
    alpha, beta = -1.25, 0.5

    # existing entry point (segmented path, scratch from the allocator)
    y_ref = torch.from_numpy(y0).cuda()
    G.spmv(x, y_ref, alpha=alpha, beta=beta)
    torch.cuda.synchronize()
    y_ref = y_ref.cpu().numpy()
    scale = orc.spmv_bound(R, x.cpu().numpy(), y0, alpha=alpha, beta=beta)

    # the no-alloc entry point, with an allocator that fails and counts calls
    calls = {"alloc": 0, "free": 0}

    def fail_alloc(nbytes, stream, ctx):
        calls["alloc"] += 1
        return None

    def count_free(ptr, stream, ctx):
        calls["free"] += 1

    a_cb, f_cb = ALLOC_FN(fail_alloc), FREE_FN(count_free)
    assert L.amgt_set_allocator(ctypes.cast(a_cb, ctypes.c_void_p), ctypes.cast(f_cb, ctypes.c_void_p), None) == 0
    try:
        outs = []
        for _ in range(2):
            y = torch.from_numpy(y0).cuda()
            torch.cuda.synchronize()
            assert _spmv_noalloc(L, 0, alpha, G, x, beta, y) == 0
            torch.cuda.synchronize()
            outs.append(y.cpu().numpy())
    finally:
        assert L.amgt_set_allocator(None, None, None) == 0
    assert calls == {"alloc": 0, "free": 0}
    # against the oracle's mBSR SpMV directly (not only the allocating path,
    # which runs the same two kernels), and against the allocating path
    y_orc = orc.spmv(R, x.cpu().numpy(), y0, alpha=alpha, beta=beta)
    for y in outs:
        assert np.all(np.abs(y - y_orc) <= 1e-12 * scale + 1e-300)
        assert np.all(np.abs(y - y_ref) <= 1e-12 * scale + 1e-300)


def test_noalloc_spmv_matrix_without_blocks_scales_y(amgt, orc):
    """Rows but no stored block: y = beta * y, as amgt_spmv gives."""
    L = amgt.lib()
    m, n = 37, 21
    E = orc.CSR(m, n, np.zeros(m + 1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    G = amgt.Bsr.from_csr(*to_dev(E))
    G.balance()
    assert G.s.blc_num == 0
    x = torch.ones(n, dtype=torch.float64, device="cuda")
    y0 = orc.rand_uniform(51, m)
    for beta in (0.75, 0.0):
        outs = []
        for _ in range(2):
            y = torch.from_numpy(y0).cuda()
            assert _spmv_noalloc(L, 0, 2.0, G, x, beta, y) == 0
            outs.append(y.cpu().numpy())
        y_ref = torch.from_numpy(y0).cuda()
        G.spmv(x, y_ref, alpha=2.0, beta=beta)
        for y in outs:
            np.testing.assert_array_equal(y, y_ref.cpu().numpy())
            np.testing.assert_array_equal(y, beta * y0)


def test_noalloc_spmv_reduced_precision(amgt, orc):
    L = amgt.lib()
    A = random_csr(orc, 300, 30000, 8, seed=22, dense_rows={7: 4000, 150: 2000})
    G = amgt.Bsr.from_csr(*to_dev(A))
    G.balance()
    G.make_shadow(amgt.FLOAT)
    x = torch.from_numpy(orc.rand_uniform(41, A.n)).cuda()
    y_ref = G.spmv(x, prec=amgt.FLOAT)
    y = torch.zeros(A.m, dtype=torch.float64, device="cuda")
    assert _spmv_noalloc(L, amgt.FLOAT, 1.0, G, x, 0.0, y) == 0
    R = orc.csr2bsr(A)
    scale = orc.spmv_bound(R, x.cpu().numpy(), None)
    assert np.all(np.abs(y.cpu().numpy() - y_ref.cpu().numpy()) <= 1e-5 * scale + 1e-300)


def test_noalloc_rejects_too_many_segments_and_missing_table(amgt, orc):
    L = amgt.lib()
    nseg = amgt._lib.NOALLOC_MAX_SEGMENTS + 1
    n = 4 * nseg
    idx = torch.arange(n + 1, dtype=torch.int32, device="cuda")
    G = amgt.Bsr.from_csr(n, n, idx, idx[:-1].contiguous(), torch.ones(n, dtype=torch.float64, device="cuda"))
    x = torch.ones(n, dtype=torch.float64, device="cuda")
    y = torch.zeros(n, dtype=torch.float64, device="cuda")
    assert _spmv_noalloc(L, 0, 1.0, G, x, 0.0, y) == 1  # no segment table yet
    G.balance()
    assert G.s.warpnum == nseg
    assert _spmv_noalloc(L, 0, 1.0, G, x, 0.0, y) == 7  # AMGT_ERR_TOO_LARGE
    assert L.amgt_status_string(7) == b"size exceeds the fixed maximum of this entry point"
