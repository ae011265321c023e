"""GPU tests of the batching form.

Many right-hand sides on one hierarchy (amgt_amg_solve_multi, every cycle
operator one tensor-core SpMM over all columns): each column's residual,
checked in fp64 by the oracle, is <= 1e-8, and each column's x agrees with
the oracle's fp64 AMG-PCG solution of that right-hand side to 1e-6 relative
(both stop at 1e-8).

Uneven systems in one launch (amgt_batch_setup + amgt_amg_solve_batch):
every system reaches its own 1e-8 (checked in fp64 by the oracle), takes
the same number of PCG iterations as the oracle's AMG-PCG on that system
alone, and its x agrees with the oracle's to 1e-8 relative; graph and
direct launches give the same bits."""
import numpy as np
import pytest
import torch

from gpu_util import to_dev

pytestmark = pytest.mark.gpu


def _multi(amgt, orc, dims, nv, policy, inner_prec0):
    from amgt_b200.amg import AmgSolver, default_params

    A = orc.laplacian(*dims)
    Ps = orc.geometric_hierarchy(*dims)
    B = np.ascontiguousarray(np.stack([orc.rand_uniform(v, A.n) for v in range(nv)], axis=1))
    amgt.set_level_policy(policy)
    try:
        S = AmgSolver(to_dev(A), [to_dev(P) for P in Ps],
                      default_params(inner_prec0=inner_prec0, galerkin_by_level=1 if policy != [0] else 0))
        X, its, rel = S.solve_multi(torch.from_numpy(B).cuda())
        S.free()
    finally:
        amgt.set_level_policy([])
    X = X.cpu().numpy()
    Sa = A.to_scipy()
    H = orc.Amg(A, Ps)
    errs = []
    for v in range(nv):
        assert rel[v] <= 1e-8
        assert np.linalg.norm(B[:, v] - Sa @ X[:, v]) <= 1.0000001e-8 * np.linalg.norm(B[:, v])
        xo, _, _, _ = H.solve(B[:, v])
        errs.append(np.linalg.norm(X[:, v] - xo) / np.linalg.norm(xo))
    assert max(errs) <= 1e-6
    assert all(0 < k <= 60 for k in its)
    return its, errs


@pytest.mark.parametrize("policy,inner", [([0], 0), ([0, 1, 1, 2], 1)])
def test_multi_rhs_small(amgt, orc, policy, inner):
    _multi(amgt, orc, (24, 22, 20), 8, policy, inner)


def test_multi_rhs_64cubed_32_rhs_tensor_cores(amgt, orc):
    """C4a: 7-point 64^3, 32 right-hand sides (seeds 0..31), levels 1-2
    fp32 and >= 3 fp16 on the tensor cores, level 0 inside the correction
    in fp32, fp64 residuals."""
    its, errs = _multi(amgt, orc, (64, 64, 64), 32, [0, 1, 1, 2], 1)
    print(f"C4a: iterations per column {min(its)}..{max(its)}, max error vs fp64 oracle {max(errs):.2e}")


def _systems(orc, sides):
    out = []
    for n in sides:
        A = orc.laplacian(int(n), int(n), 1)
        out.append((A, orc.geometric_hierarchy(int(n), int(n), 1)))
    return out


def _batch(amgt, systems, **kw):
    from amgt_b200.amg import BatchSolver, default_params

    return BatchSolver([(to_dev(A), [to_dev(P) for P in Ps]) for A, Ps in systems], default_params(**kw))


def _check_batch(amgt, orc, sides, exact_iters=True):
    amgt.set_level_policy([0])
    try:
        systems = _systems(orc, sides)
        S = _batch(amgt, systems)
        b = np.concatenate([orc.rand_uniform(i, A.n) for i, (A, _) in enumerate(systems)])
        x, its, rel, loop_it = S.solve_batch(torch.from_numpy(b).cuda())
        off = S.offsets
        S.free()
    finally:
        amgt.set_level_policy([])
    x = x.cpu().numpy()
    assert loop_it == max(its)
    for i, (A, Ps) in enumerate(systems):
        xs, bs = x[off[i]:off[i + 1]], b[off[i]:off[i + 1]]
        assert rel[i] <= 1e-8
        assert np.linalg.norm(bs - A.to_scipy() @ xs) <= 1.0000001e-8 * np.linalg.norm(bs)
        xo, it_o, _, _ = orc.Amg(A, Ps).solve(bs)
        if exact_iters:
            assert its[i] == it_o, (i, sides[i])
        else:
            assert abs(its[i] - it_o) <= 1, (i, sides[i])
        assert np.linalg.norm(xs - xo) <= 1e-8 * np.linalg.norm(xo)
    return its


def test_batch_uneven_small_matches_oracle_per_system(amgt, orc):
    _check_batch(amgt, orc, [9, 17, 32, 45, 64, 70, 96, 23, 50, 81])


def test_batch_64_systems_sides_32_to_512(amgt, orc):
    """C4b: 64 independent 2D 5-point Poisson systems, sides uniform in
    [32, 512] (seed 0), one graph launch for the whole solve."""
    sides = np.random.default_rng(0).integers(32, 513, size=64)
    its = _check_batch(amgt, orc, list(sides), exact_iters=False)
    print(f"C4b: {sum(int(s) ** 2 for s in sides):,} rows, iterations per system {min(its)}..{max(its)}")


def test_batch_graph_and_direct_agree(amgt, orc):
    systems = _systems(orc, [12, 40, 33])
    b = torch.from_numpy(np.concatenate([orc.rand_uniform(i, A.n) for i, (A, _) in enumerate(systems)])).cuda()
    outs = []
    for g in (1, 0):
        S = _batch(amgt, systems, use_graph=g)
        x, its, rel, k = S.solve_batch(b)
        outs.append((x.clone(), its, rel, k))
        x2, its2, rel2, k2 = S.solve_batch(b)  # a second solve reuses the graph
        assert torch.equal(x2, x) and its2 == its
        S.free()
    assert torch.equal(outs[0][0], outs[1][0]) and outs[0][1:] == outs[1][1:]
