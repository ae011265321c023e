"""CPU tests of the policy's oracle (the numpy restatement the GPU kernels
are checked against): the MLP gradient against central finite differences,
and the structured interpolation against the geometric one."""
import numpy as np

from oracle import mlp_oracle as mo


def test_mlp_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.3, mo.NPARAM)
    X = rng.normal(0, 1, (7, 16))
    T = np.stack([rng.uniform(0, 1, 7), rng.integers(0, 3, 7)], axis=1)
    g = mo.grad(p, X, T)
    idx = rng.choice(mo.NPARAM, 60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros(mo.NPARAM)
        e[i] = h
        fd = (mo.loss(p + e, X, T) - mo.loss(p - e, X, T)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), i


def test_structured_interp_full_coarsening_equals_geometric():
    from amgt_b200 import problems

    for dims in ((9, 7, 5), (8, 6, 1), (5, 1, 1)):
        (m, n, ia, ja, a), cd = problems.interp(*dims)
        D = np.zeros((m, n))
        for r in range(m):
            D[r, ja[ia[r]:ia[r + 1]]] = a[ia[r]:ia[r + 1]]
        np.testing.assert_array_equal(mo.structured_interp(dims, (1, 1, 1)), D)


def test_structured_interp_semicoarsening_rows_sum_to_one():
    # odd extents: every fine point has both coarse neighbours (with an even
    # extent the last point has one, weight 1/2, as in problems.interp)
    P = mo.structured_interp((9, 7, 4), (0, 1, 0))
    assert P.shape == (252, 9 * 4 * 4)
    np.testing.assert_allclose(P.sum(axis=1), 1.0)


def test_aniso_problem_is_symmetric_and_anisotropic():
    n, _, ia, ja, a = mo.aniso_problem((7, 6, 1), 1e-2, 0.3)
    D = np.zeros((n, n))
    for r in range(n):
        D[r, ja[ia[r]:ia[r + 1]]] = a[ia[r]:ia[r + 1]]
    np.testing.assert_allclose(D, D.T, atol=1e-15)
    assert np.all(np.linalg.eigvalsh(D) > 0)
