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


def test_committed_network_fits_its_training_set():
    """The trained weights (amgt_b200/data/policy_mlp.npy, trained on the
    GPU by amgt_mlp_train) against the committed dataset, evaluated by the
    oracle's forward pass: the loss is far below the initial network's, and
    the theta it predicts tracks the labels."""
    import os

    import amgt_b200.policy as pol

    d = np.load(os.path.join(os.path.dirname(pol.WEIGHTS), "policy_dataset.npz"))
    X, T = d["X"], d["T"]
    assert X.shape[1] == 16 and T.shape == (X.shape[0], 2) and X.shape[0] > 20000
    assert set(np.unique(T[:, 1])) <= {0.0, 1.0, 2.0}
    w = np.load(pol.WEIGHTS)
    rng = np.random.default_rng(0)
    w0 = np.zeros(mo.NPARAM, np.float32)
    o = 0
    for fan_in, fan_out in ((16, 64), (64, 64), (64, 4)):  # the initialisation train() uses
        n = fan_out * fan_in
        w0[o:o + n] = rng.normal(0.0, np.sqrt(2.0 / fan_in), size=n)
        o += n + fan_out
    trained, initial = mo.loss(w, X, T), mo.loss(w0, X, T)
    assert trained < 0.2 * initial
    _, _, out = mo.forward(w, X)
    theta = 1.0 / (1.0 + np.exp(-out[:, 0]))
    assert np.corrcoef(theta, T[:, 0])[0, 1] > 0.8
