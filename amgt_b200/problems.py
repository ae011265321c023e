"""Seeded synthetic problems (host, numpy): the inputs the bench and the
solver feed to the kernels.

Structured operators follow HYPRE's generators: unknowns ordered x fastest
(row = x + nx*(y + ny*z)), the diagonal stored first and the other columns
ascending (GenerateLaplacian, AmgT_HYPRE/src/parcsr_ls/par_laplace.c:15;
GenerateLaplacian27pt, par_laplace_27pt.c:15; GenerateLaplacian9pt,
par_laplace_9pt.c:15; stencil values as in AmgT_HYPRE/src/test/ij_mm.c).
"""
from __future__ import annotations

import numpy as np

_PHI = np.uint64(0x9E3779B97F4A7C15)


def _mix64(z: np.ndarray) -> np.ndarray:
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def rand_u64(seed: int, k: np.ndarray) -> np.ndarray:
    """Counter-based stream: splitmix64 finaliser of seed*phi + k + 1."""
    with np.errstate(over="ignore"):
        return _mix64(np.uint64(seed) * _PHI + k.astype(np.uint64) + np.uint64(1))


def rand_uniform(seed: int, n: int) -> np.ndarray:
    """n values uniform in [-1, 1) (53 random bits each)."""
    u = rand_u64(seed, np.arange(n, dtype=np.uint64)) >> np.uint64(11)
    return u.astype(np.float64) * (2.0 / 9007199254740992.0) - 1.0


def _grid(nx, ny, nz):
    r = np.arange(nx * ny * nz, dtype=np.int64)
    return r, r % nx, (r // nx) % ny, r // (nx * ny)


def _assemble(n, cols, vals, valid):
    """Rows of candidate (col, val) in storage order -> CSR keeping order."""
    lens = valid.sum(axis=1)
    ia = np.zeros(n + 1, np.int32)
    np.cumsum(lens, out=ia[1:])
    return ia, cols[valid].astype(np.int32), vals[valid].astype(np.float64)


def laplacian(nx: int, ny: int, nz: int, cx=1.0, cy=1.0, cz=1.0):
    """7-point (5-point when nz == 1) Laplacian; returns (n, n, ia, ja, a)."""
    n = nx * ny * nz
    r, x, y, z = _grid(nx, ny, nz)
    sxy = nx * ny
    diag = (2.0 * cx if nx > 1 else 0.0) + (2.0 * cy if ny > 1 else 0.0) + (2.0 * cz if nz > 1 else 0.0)
    cols = np.stack([r, r - sxy, r - nx, r - 1, r + 1, r + nx, r + sxy], axis=1)
    vals = np.broadcast_to(np.array([diag, -cz, -cy, -cx, -cx, -cy, -cz]), (n, 7))
    valid = np.stack([np.ones(n, bool), z > 0, y > 0, x > 0, x < nx - 1, y < ny - 1, z < nz - 1], axis=1)
    return (n, n) + _assemble(n, cols, vals, valid)


def _box_offsets():
    return [(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1) if (dx, dy, dz) != (0, 0, 0)]


def box(nx: int, ny: int, nz: int):
    """27-point (9-point when nz == 1) Laplacian: diagonal 26 (8), off -1."""
    n = nx * ny * nz
    r, x, y, z = _grid(nx, ny, nz)
    diag = 26.0 if nz > 1 else (8.0 if ny > 1 else 2.0)
    offs = _box_offsets()
    cols = [r]
    valid = [np.ones(n, bool)]
    for dx, dy, dz in offs:
        cols.append(r + dx + dy * nx + dz * nx * ny)
        valid.append((x + dx >= 0) & (x + dx < nx) & (y + dy >= 0) & (y + dy < ny) & (z + dz >= 0) & (z + dz < nz))
    cols = np.stack(cols, axis=1)
    valid = np.stack(valid, axis=1)
    vals = np.full(cols.shape, -1.0)
    vals[:, 0] = diag
    return (n, n) + _assemble(n, cols, vals, valid)


def varcoef27(nx: int, ny: int, nz: int, seed: int = 1, sigma: float = 2.0, ratio: float = 1e3):
    """27-point variable-coefficient diffusion: node coefficient
    k = exp(sigma * N(0,1)) clipped to max/min <= ratio; coupling
    -w * 2 k_i k_j / (k_i + k_j) with w = 1 (face), 1/2 (edge), 1/4 (corner);
    diagonal = sum of all 26 couplings, an out-of-domain neighbour counting
    with k_j = k_i (Dirichlet).  Symmetric positive definite."""
    n = nx * ny * nz
    r, x, y, z = _grid(nx, ny, nz)
    k2 = np.arange(n, dtype=np.uint64) * np.uint64(2)
    u1 = ((rand_u64(seed, k2) >> np.uint64(11)).astype(np.float64) + 1.0) / 9007199254740993.0
    u2 = (rand_u64(seed, k2 + np.uint64(1)) >> np.uint64(11)).astype(np.float64) / 9007199254740992.0
    g = np.sqrt(-2.0 * np.log(u1)) * np.cos(6.283185307179586 * u2)
    clip = 0.5 * np.log(ratio)
    kap = np.exp(np.clip(sigma * g, -clip, clip))
    cols = [r]
    vals = [np.zeros(n)]
    valid = [np.ones(n, bool)]
    diag = np.zeros(n)
    for dx, dy, dz in _box_offsets():
        m = (dx != 0) + (dy != 0) + (dz != 0)
        w = 1.0 if m == 1 else (0.5 if m == 2 else 0.25)
        inside = (x + dx >= 0) & (x + dx < nx) & (y + dy >= 0) & (y + dy < ny) & (z + dz >= 0) & (z + dz < nz)
        c = r + dx + dy * nx + dz * nx * ny
        kj = np.where(inside, kap[np.where(inside, c, r)], kap)
        h = w * 2.0 * kap * kj / (kap + kj)
        diag += h
        cols.append(c)
        vals.append(-h)
        valid.append(inside)
    vals[0] = diag
    return (n, n) + _assemble(n, np.stack(cols, 1), np.stack(vals, 1), np.stack(valid, 1))


def _interp_1d(i: np.ndarray, nfine: int, ncoarse: int):
    """Up to two (coarse index, weight) pairs per fine index."""
    if nfine == 1:
        z = np.zeros_like(i)
        return [(z, np.ones(i.shape), np.ones(i.shape, bool)), (z, np.zeros(i.shape), np.zeros(i.shape, bool))]
    even = (i & 1) == 0
    c0 = np.where(even, i // 2, (i - 1) // 2)
    w0 = np.where(even, 1.0, 0.5)
    c1 = (i + 1) // 2
    v1 = (~even) & (c1 < ncoarse)
    return [(c0, w0, np.ones(i.shape, bool)), (np.where(v1, c1, 0), np.where(v1, 0.5, 0.0), v1)]


def interp(nx: int, ny: int, nz: int):
    """Linear interpolation between vertex-centred grids (coarse point j on
    fine point 2j, tensor product over the dimensions with extent > 1).
    Returns ((m, nc, ia, ja, a), (ncx, ncy, ncz)); rows sorted."""
    ncx = (nx + 1) // 2 if nx > 1 else 1
    ncy = (ny + 1) // 2 if ny > 1 else 1
    ncz = (nz + 1) // 2 if nz > 1 else 1
    n = nx * ny * nz
    r, x, y, z = _grid(nx, ny, nz)
    px, py, pz = _interp_1d(x, nx, ncx), _interp_1d(y, ny, ncy), _interp_1d(z, nz, ncz)
    cols, vals, valid = [], [], []
    for c in range(2):
        for b in range(2):
            for q in range(2):
                cols.append(px[q][0] + ncx * (py[b][0] + ncy * pz[c][0]))
                vals.append(px[q][1] * py[b][1] * pz[c][1])
                valid.append(px[q][2] & py[b][2] & pz[c][2])
    ia, ja, a = _assemble(n, np.stack(cols, 1), np.stack(vals, 1), np.stack(valid, 1))
    return (n, ncx * ncy * ncz, ia, ja, a), (ncx, ncy, ncz)


def csr_transpose(m: int, n: int, ia: np.ndarray, ja: np.ndarray, a: np.ndarray):
    """Host CSR transpose with sorted rows (used to state R = P^T inputs)."""
    rows = np.repeat(np.arange(m, dtype=np.int64), np.diff(ia))
    order = np.lexsort((rows, ja))
    tia = np.zeros(n + 1, np.int32)
    np.cumsum(np.bincount(ja, minlength=n), out=tia[1:])
    return n, m, tia, rows[order].astype(np.int32), a[order]
