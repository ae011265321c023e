"""CPU restatement (numpy, float64) of the policy MLP's forward pass, loss
and gradient, of the level features and of the structured interpolation --
test infrastructure only: the tests compare the CUDA kernels of
amgt_b200/csrc/policy.cu against these, and check these gradients against
finite differences.

The parameter layout, loss and feature definitions follow the kernels'
documented contract (include/amgt_b200.h, "learned precision / theta
policy"); there is no reference counterpart (AmgT fixes its level ->
precision table, AmgT_HYPRE/src/seq_mv/csr_spgemm_device.c:1847-1862).
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 16, 64, 4
NPARAM = HID * IN + HID + HID * HID + HID + OUT * HID + OUT


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    W1 = p[o:o + HID * IN].reshape(HID, IN); o += HID * IN
    b1 = p[o:o + HID]; o += HID
    W2 = p[o:o + HID * HID].reshape(HID, HID); o += HID * HID
    b2 = p[o:o + HID]; o += HID
    W3 = p[o:o + OUT * HID].reshape(OUT, HID); o += OUT * HID
    b3 = p[o:o + OUT]
    return W1, b1, W2, b2, W3, b3


def forward(p, X):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    z1 = X @ W1.T + b1
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0.0)
    o = h2 @ W3.T + b3
    return h1, h2, o


def loss(p, X, T):
    _, _, o = forward(p, X)
    sg = 1.0 / (1.0 + np.exp(-o[:, 0]))
    lg = o[:, 1:4]
    lg = lg - lg.max(axis=1, keepdims=True)
    logp = lg - np.log(np.exp(lg).sum(axis=1, keepdims=True))
    cls = T[:, 1].astype(np.int64)
    return float(np.mean((sg - T[:, 0]) ** 2 - logp[np.arange(len(cls)), cls]))


def grad(p, X, T):
    """Mean gradient of the loss over the samples (flat, the kernel's
    layout)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    h1, h2, o = forward(p, X)
    n = X.shape[0]
    sg = 1.0 / (1.0 + np.exp(-o[:, 0]))
    lg = o[:, 1:4] - o[:, 1:4].max(axis=1, keepdims=True)
    sm = np.exp(lg) / np.exp(lg).sum(axis=1, keepdims=True)
    dO = np.zeros((n, OUT))
    dO[:, 0] = 2.0 * (sg - T[:, 0]) * sg * (1.0 - sg)
    onehot = np.zeros((n, 3))
    onehot[np.arange(n), T[:, 1].astype(np.int64)] = 1.0
    dO[:, 1:4] = sm - onehot
    dW3 = dO.T @ h2 / n
    db3 = dO.mean(axis=0)
    dh2 = (dO @ W3) * (h2 > 0)
    dW2 = dh2.T @ h1 / n
    db2 = dh2.mean(axis=0)
    dh1 = (dh2 @ W2) * (h1 > 0)
    dW1 = dh1.T @ X / n
    db1 = dh1.mean(axis=0)
    return np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])


def structured_interp(dims, coarsen):
    """Dense restatement of amgt_structured_interp: P = Px (x) Py (x) Pz with
    linear interpolation (coarse j on fine 2j) along coarsened axes."""
    mats = []
    for d in range(3):
        nf = dims[d]
        if coarsen[d] and nf > 1:
            nc = (nf + 1) // 2
            M = np.zeros((nf, nc))
            for i in range(nf):
                if i % 2 == 0:
                    M[i, i // 2] = 1.0
                else:
                    M[i, (i - 1) // 2] = 0.5
                    if (i + 1) // 2 < nc:
                        M[i, (i + 1) // 2] = 0.5
        else:
            M = np.eye(nf)
        mats.append(M)
    # x fastest: row = x + nx (y + ny z)  ->  kron(Pz, kron(Py, Px))
    return np.kron(mats[2], np.kron(mats[1], mats[0]))


def features(A_dense, level, dims):
    """Restatement of amgt_level_features on a dense operator."""
    A = np.asarray(A_dense, np.float64)
    n = A.shape[0]
    nx, ny, nz = dims
    dd, rsn, npos, noff, sx, sy, sz, mix, omax = [], [], 0, 0, 0.0, 0.0, 0.0, 0.0, []
    for i in range(n):
        cols = np.nonzero(A[i])[0]
        d = A[i, i]
        ad = abs(d) if d != 0 else 1.0
        off = [c for c in cols if c != i]
        offs = np.abs(A[i, off]).sum() if off else 0.0
        dd.append(min(abs(d) / offs, 10.0) if offs > 0 else 10.0)
        rsn.append(A[i, cols].sum() / ad)
        om = 0.0
        for c in off:
            a = A[i, c]
            npos += a > 0
            noff += 1
            om = max(om, abs(a))
            o = int(c - i)
            sxy = nx * ny  # nearest multiple, halves away from zero (the kernel's integer rule)
            z = (o + sxy // 2) // sxy if o >= 0 else -((-o + sxy // 2) // sxy)
            o -= z * sxy
            y = (o + nx // 2) // nx if o >= 0 else -((-o + nx // 2) // nx)
            x = o - y * nx
            if x:
                sx += abs(a) / ad
            if y:
                sy += abs(a) / ad
            if z:
                sz += abs(a) / ad
            if (x != 0) + (y != 0) + (z != 0) > 1:
                mix += abs(a) / ad
        omax.append(om / ad)
    nnz = np.count_nonzero(A)
    den = sx + sy + sz if sx + sy + sz > 0 else 1.0
    rsn = np.array(rsn)
    return np.array([np.log10(n), nnz / n / 10.0, np.nan, np.mean(dd), np.min(dd), rsn.mean(),
                     np.sqrt(max(0.0, (rsn ** 2).mean() - rsn.mean() ** 2)), npos / noff if noff else 0.0,
                     sx / den, sy / den, sz / den, mix / den, np.mean(omax), level / 10.0, 1.0 if nz > 1 else 0.0,
                     1.0])


def aniso_problem(dims, eps, angle):
    """Restatement of amgt_aniso_problem: (n, n, ia, ja, a), diagonal first
    then ascending columns."""
    nx, ny, nz = dims
    cs, sn = np.cos(angle), np.sin(angle)
    a = cs * cs + eps * sn * sn
    b = (1.0 - eps) * cs * sn
    c = sn * sn + eps * cs * cs
    ia, ja, va = [0], [], []
    for r in range(nx * ny * nz):
        x, y, z = r % nx, (r // nx) % ny, r // (nx * ny)
        cols, vals = [r], [2 * a + 2 * c + (2.0 if nz > 1 else 0.0)]
        if z > 0:
            cols.append(r - nx * ny); vals.append(-1.0)
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if (dx, dy) == (0, 0) or not (0 <= x + dx < nx and 0 <= y + dy < ny):
                    continue
                v = -a if dy == 0 else (-c if dx == 0 else (-0.5 * b if dx == dy else 0.5 * b))
                if v == 0.0:
                    continue
                cols.append(r + dx + dy * nx); vals.append(v)
        if z + 1 < nz:
            cols.append(r + nx * ny); vals.append(-1.0)
        ja += cols
        va += vals
        ia.append(len(ja))
    n = nx * ny * nz
    return n, n, np.array(ia, np.int32), np.array(ja, np.int32), np.array(va)
