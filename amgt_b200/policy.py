"""Learned per-level precision / strength-threshold policy.

A hierarchy is built level by level through amgt_amg_setup_adaptive: at
level l the library hands over A_l, the policy reads 16 features of A_l
(amgt_level_features, on the GPU), picks level l's precision and a strength
threshold theta, and theta picks the coarsening: grid axis d is coarsened
when its share of the off-diagonal coupling is at least theta times the
largest share (structured semi-coarsening with linear interpolation,
amgt_structured_interp; theta = 0 coarsens every axis, as geometric
full coarsening does).  This is the place BoomerAMG's strength threshold
(HYPRE_BoomerAMGSetStrongThreshold) and the level -> precision table
(get_calculationPrecison, AmgT_HYPRE/src/seq_mv/csr_spgemm_device.c:
1847-1862) take in the reference.

Policies:
  FixedPolicy  theta and a precision table: the plain FP64 configuration
               (theta 0.25, every level fp64) is the fallback and the yardstick;
  MLPPolicy    the 16 -> 64 -> 64 -> 4 MLP (amgt_mlp_forward) on the level's
               features: theta = sigmoid(output 0), precision = argmax of
               outputs 1..3 (fp64 / fp32 / fp16); level 0 stays fp64 (its
               residual is the solve's fp64 residual).

make_dataset labels seeded rotated-anisotropic problems with the plain
solver's convergence (theta* = the candidate with the least work, iterations
times operator complexity; a level's class = the narrowest precision whose
use on every coarse level takes no more iterations than fp64), and train()
fits the MLP on the GPU with the library's own kernels (amgt_mlp_train).
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np
import torch

from . import _lib as L
from ._lib import AmgtAmgParams, AmgtBsr, AmgtCsr, check
from .amg import AmgSolver, default_params
from .mbsr import _stream, csr_struct

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "data", "policy_mlp.npy")
NPARAM = 5508
THETAS = (0.05, 0.25, 0.5, 0.75)
PREC_OF_CLASS = (L.DOUBLE, L.FLOAT, L.HALF)

COARSEN_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_int, ctypes.POINTER(AmgtBsr), ctypes.POINTER(AmgtCsr),
                              ctypes.POINTER(ctypes.c_int), ctypes.c_void_p)


def level_features(A: AmgtBsr, level: int, dims, stream=None) -> np.ndarray:
    out = (ctypes.c_float * 16)()
    d = (ctypes.c_int * 3)(*dims)
    check(L.lib().amgt_level_features(ctypes.byref(A), level, d, out, _stream(stream)), "amgt_level_features")
    return np.array(out[:], dtype=np.float32)


def coarsen_axes(feats: np.ndarray, dims, theta: float):
    """Axes to coarsen: extent > 2 and coupling share >= theta * the largest
    such share."""
    share = [float(feats[8]), float(feats[9]), float(feats[10])]
    ok = [dims[d] > 2 for d in range(3)]
    smax = max([share[d] for d in range(3) if ok[d]], default=0.0)
    if smax <= 0.0:
        return [int(ok[d]) for d in range(3)]
    return [int(ok[d] and share[d] >= theta * smax) for d in range(3)]


class FixedPolicy:
    def __init__(self, theta: float = 0.25, precs=(L.DOUBLE,)):
        self.theta, self.precs = theta, list(precs)

    def decide(self, level: int, feats: np.ndarray):
        return self.theta, self.precs[min(level, len(self.precs) - 1)]


class MLPPolicy:
    def __init__(self, params: torch.Tensor):
        if not (params.is_cuda and params.dtype == torch.float32 and params.numel() == NPARAM):
            raise TypeError("params: 5508 float32 CUDA values")
        self.params = params.contiguous()
        self._x = torch.zeros(16, dtype=torch.float32, device="cuda")
        self._o = torch.zeros(4, dtype=torch.float32, device="cuda")

    @classmethod
    def load(cls, path: str = WEIGHTS) -> "MLPPolicy":
        return cls(torch.from_numpy(np.load(path).astype(np.float32)).cuda())

    def outputs(self, feats: np.ndarray) -> np.ndarray:
        self._x.copy_(torch.from_numpy(np.asarray(feats, np.float32)))
        check(L.lib().amgt_mlp_forward(self.params.data_ptr(), 1, self._x.data_ptr(), self._o.data_ptr(),
                                       _stream(None)), "amgt_mlp_forward")
        return self._o.cpu().numpy()

    def decide(self, level: int, feats: np.ndarray):
        o = self.outputs(feats)
        theta = 1.0 / (1.0 + math.exp(-float(o[0])))
        prec = L.DOUBLE if level == 0 else PREC_OF_CLASS[int(np.argmax(o[1:4]))]
        return theta, prec


class AdaptiveSolver(AmgSolver):
    """Hierarchy built level by level by a policy (amgt_amg_setup_adaptive).
    A: device CSR tuple; dims: its grid.  trace: per level (features,
    theta, precision, coarsened axes)."""

    def __init__(self, A, dims, policy, params: AmgtAmgParams | None = None, coarse_rows: int = 64,
                 max_levels: int = 25, stream=None):
        m, n, ia, ja, a = A
        self._keep = [A]
        self._A = csr_struct(m, n, ia, ja, a)
        self.params = params if params is not None else default_params()
        self.params.max_levels = max_levels
        self.trace = []
        Ps = []
        state = {"dims": list(dims), "err": None}

        def cb(level, Ap, Pp, precp, ctx):
            try:
                Al = Ap.contents
                d = state["dims"]
                f = level_features(Al, level, d, stream)
                theta, prec = policy.decide(level, f)
                precp[0] = int(prec)
                axes = coarsen_axes(f, d, theta)
                stop = Al.row <= coarse_rows or not any(axes)
                self.trace.append({"level": level, "rows": int(Al.row), "dims": list(d), "features": f,
                                   "theta": float(theta), "prec": int(prec), "axes": axes if not stop else None})
                if stop:
                    return 1
                P = AmgtCsr()
                cd = (ctypes.c_int * 3)()
                check(L.lib().amgt_structured_interp((ctypes.c_int * 3)(*d), (ctypes.c_int * 3)(*axes),
                                                     ctypes.byref(P), cd, _stream(stream)), "amgt_structured_interp")
                Ps.append(P)
                Pp[0] = P
                state["dims"] = list(cd[:])
                return 0
            except Exception as e:  # noqa: BLE001 - reported after the setup returns
                state["err"] = e
                return -1

        fn = COARSEN_FN(cb)
        self.h = ctypes.c_void_p()
        try:
            rc = L.lib().amgt_amg_setup_adaptive(ctypes.byref(self._A), ctypes.cast(fn, ctypes.c_void_p), None,
                                                 ctypes.byref(self.params), ctypes.byref(self.h), _stream(stream))
        finally:
            for P in Ps:
                L.lib().amgt_csr_free(ctypes.byref(P), _stream(stream))
        if state["err"] is not None:
            raise state["err"]
        check(rc, "amgt_amg_setup_adaptive")
        self.n = m

    def operator_complexity(self) -> float:
        nnz = [self.level(l)["nnz"] for l in range(self.num_levels())]
        return sum(nnz) / nnz[0]


def aniso_problem(dims, eps: float, angle: float, stream=None):
    """Rotated anisotropic diffusion (amgt_aniso_problem) as a device CSR
    tuple of torch tensors (copies; the library's arrays are freed)."""
    c = AmgtCsr()
    check(L.lib().amgt_aniso_problem((ctypes.c_int * 3)(*dims), eps, angle, ctypes.byref(c), _stream(None)),
          "amgt_aniso_problem")
    from .mbsr import view

    try:
        out = (c.num_rows, c.num_cols, view(c.i, c.num_rows + 1, torch.int32).clone(),
               view(c.j, c.num_nonzeros, torch.int32).clone(), view(c.data, c.num_nonzeros, torch.float64).clone())
    finally:
        L.lib().amgt_csr_free(ctypes.byref(c), _stream(None))
    return out


def problem_params(seed: int, held_out: bool = False):
    """Seeded training problem: 2D or 3D, anisotropy eps log-uniform in
    [1e-3, 1], angle uniform in [0, pi), unknowns log-uniform in 32^2 ..
    64^3 (held-out problems: 128^3)."""
    rng = np.random.default_rng(seed)
    eps = float(10.0 ** rng.uniform(-3.0, 0.0))
    angle = float(rng.uniform(0.0, math.pi))
    if held_out:
        return (128, 128, 128), eps, angle
    three_d = bool(rng.integers(0, 2))
    nrows = float(np.exp(rng.uniform(math.log(32 ** 2), math.log(64 ** 3))))
    if three_d:
        s = int(min(64, max(12, round(nrows ** (1 / 3)))))
        return (s, s, s), eps, angle
    s = int(min(512, max(32, round(math.sqrt(nrows)))))
    return (s, s, 1), eps, angle


def solve_with(A, dims, b, policy, **kw):
    """(iterations, relative residual, operator complexity, trace, x, setup s,
    solve s) of PCG + V(1,1) on the hierarchy the policy builds."""
    import time

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    S = AdaptiveSolver(A, dims, policy, default_params(**kw))
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    x, it, rel = S.solve(b)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    oc = S.operator_complexity()
    trace = S.trace
    S.free()
    return {"iters": it, "relres": rel, "complexity": oc, "trace": trace, "x": x, "setup_s": t1 - t0,
            "solve_s": t2 - t1}


def label_problem(seed: int, max_iter: int = 200):
    """Training samples of one seeded problem: per level of the theta*
    hierarchy, (features, theta*, precision class)."""
    dims, eps, angle = problem_params(seed)
    A = aniso_problem(dims, eps, angle)
    from .problems import rand_uniform

    b = torch.from_numpy(rand_uniform(seed, A[0])).cuda()
    best = None
    for th in THETAS:
        r = solve_with(A, dims, b, FixedPolicy(th), max_iter=max_iter)
        ok = r["relres"] <= 1e-8
        work = r["iters"] * r["complexity"] if ok else float("inf")
        if best is None or work < best[0]:
            best = (work, th, r)
    if not math.isfinite(best[0]):
        return None
    theta, ref = best[1], best[2]
    cls = 0
    for c, prec in ((2, L.HALF), (1, L.FLOAT)):  # narrowest first
        r = solve_with(A, dims, b, FixedPolicy(theta, (L.DOUBLE, prec)), max_iter=max_iter)
        if r["relres"] <= 1e-8 and r["iters"] <= ref["iters"]:
            cls = c
            break
    X, T = [], []
    for t in ref["trace"]:
        X.append(t["features"])
        T.append((theta, 0 if t["level"] == 0 else cls))
    return np.array(X, np.float32), np.array(T, np.float32), {"seed": seed, "dims": dims, "eps": eps, "angle": angle,
                                                              "theta": theta, "class": cls, "iters": ref["iters"]}


def make_dataset(n_problems: int = 4000, seed0: int = 0):
    Xs, Ts, meta = [], [], []
    for k in range(n_problems):
        r = label_problem(seed0 + k)
        if r is None:
            continue
        Xs.append(r[0])
        Ts.append(r[1])
        meta.append(r[2])
    return np.concatenate(Xs), np.concatenate(Ts), meta


def train(X: np.ndarray, T: np.ndarray, epochs: int = 400, batch: int = 256, lr: float = 2e-3, seed: int = 0,
          init: np.ndarray | None = None):
    """Fits the MLP on the GPU (amgt_mlp_train); returns (params, loss per
    epoch)."""
    if init is None:
        rng = np.random.default_rng(seed)
        init = np.zeros(NPARAM, np.float32)
        o = 0
        for fan_in, fan_out in ((16, 64), (64, 64), (64, 4)):
            w = rng.normal(0.0, math.sqrt(2.0 / fan_in), size=fan_out * fan_in).astype(np.float32)
            init[o:o + w.size] = w
            o += w.size + fan_out  # biases start at 0
    P = torch.from_numpy(init.copy()).cuda()
    Xd = torch.from_numpy(np.ascontiguousarray(X, np.float32)).cuda()
    Td = torch.from_numpy(np.ascontiguousarray(T, np.float32)).cuda()
    hist = (ctypes.c_float * max(1, epochs))()
    check(L.lib().amgt_mlp_train(P.data_ptr(), int(X.shape[0]), Xd.data_ptr(), Td.data_ptr(), epochs, batch, lr,
                                 seed, hist, _stream(None)), "amgt_mlp_train")
    torch.cuda.synchronize()
    return P.cpu().numpy(), np.array(hist[:epochs])
