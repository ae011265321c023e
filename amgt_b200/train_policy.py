"""Builds the learned policy: labels seeded rotated-anisotropic problems with
the plain solver (amgt_b200.policy.label_problem), trains the MLP on the GPU
(amgt_mlp_train) and evaluates it on held-out seeds against the plain FP64
configuration.

python -m amgt_b200.train_policy --problems 4000 --heldout 200 --out DIR

Writes DIR/policy_dataset.npz (features X, targets T = (theta*, class),
per-problem labels), DIR/policy_mlp.npy (the 5508 weights) and
DIR/policy_report.json (training loss, label statistics, held-out
comparison).  Training problems use seeds 0 .. problems - 1; held-out
problems use seeds 1_000_000 + k (128^3 unless --heldout-dims says
otherwise).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np


def evaluate(weights: np.ndarray, seeds, dims_override=None, max_iter=200):
    """Learned policy vs the plain FP64 configuration (theta 0.25, fp64) on
    the given seeds: iterations, convergence factor, times, and the
    learned solution's error against the fp64 one.  A learned solve that
    does not reach 1e-8 falls back to the fp64 configuration."""
    import torch

    from amgt_b200 import policy
    from amgt_b200.problems import rand_uniform

    net = policy.MLPPolicy(torch.from_numpy(weights.astype(np.float32)).cuda())
    # untimed warm-up of both configurations (module loads, pool growth)
    dims, eps, angle = policy.problem_params(seeds[0], held_out=True)
    if dims_override:
        dims = tuple(dims_override)
    A = policy.aniso_problem(dims, eps, angle)
    b = torch.ones(A[0], dtype=torch.float64, device="cuda")
    policy.solve_with(A, dims, b, policy.FixedPolicy(0.25), max_iter=max_iter)
    policy.solve_with(A, dims, b, net, max_iter=max_iter, galerkin_by_level=1)
    rows = []
    for sd in seeds:
        dims, eps, angle = policy.problem_params(sd, held_out=True)
        if dims_override:
            dims = tuple(dims_override)
        A = policy.aniso_problem(dims, eps, angle)
        b = torch.from_numpy(rand_uniform(sd, A[0])).cuda()
        ref = policy.solve_with(A, dims, b, policy.FixedPolicy(0.25), max_iter=max_iter)
        lrn = policy.solve_with(A, dims, b, net, max_iter=max_iter, galerkin_by_level=1)
        fallback = not (lrn["relres"] <= 1e-8)
        if fallback:
            lrn = dict(ref, setup_s=lrn["setup_s"] + ref["setup_s"], solve_s=lrn["solve_s"] + ref["solve_s"])
        err = float(torch.linalg.vector_norm(lrn["x"] - ref["x"]) / torch.linalg.vector_norm(ref["x"]))

        def rho(r):
            return float(r["relres"] ** (1.0 / max(1, r["iters"])))

        rows.append({"seed": sd, "dims": list(dims), "eps": eps, "angle": angle,
                     "fp64": {"iters": ref["iters"], "rho": rho(ref), "complexity": ref["complexity"],
                              "setup_s": ref["setup_s"], "solve_s": ref["solve_s"]},
                     "learned": {"iters": lrn["iters"], "rho": rho(lrn), "complexity": lrn["complexity"],
                                 "setup_s": lrn["setup_s"], "solve_s": lrn["solve_s"], "fallback": fallback,
                                 "thetas": [round(t["theta"], 3) for t in lrn["trace"]] if not fallback else None,
                                 "precs": [t["prec"] for t in lrn["trace"]] if not fallback else None},
                     "rel_err_vs_fp64": err})
    return rows


def summarize(rows):
    f = lambda k, w: [r[w][k] for r in rows]  # noqa: E731
    t64 = np.array(f("setup_s", "fp64")) + np.array(f("solve_s", "fp64"))
    tl = np.array(f("setup_s", "learned")) + np.array(f("solve_s", "learned"))
    return {"problems": len(rows),
            "fp64_mean_rho": float(np.mean(f("rho", "fp64"))), "learned_mean_rho": float(np.mean(f("rho", "learned"))),
            "fp64_mean_iters": float(np.mean(f("iters", "fp64"))),
            "learned_mean_iters": float(np.mean(f("iters", "learned"))),
            "fp64_mean_work": float(np.mean(np.array(f("iters", "fp64")) * np.array(f("complexity", "fp64")))),
            "learned_mean_work": float(np.mean(np.array(f("iters", "learned")) * np.array(f("complexity", "learned")))),
            "fp64_total_s": float(t64.sum()), "learned_total_s": float(tl.sum()),
            "speedup_total": float(t64.sum() / tl.sum()),
            "learned_faster_on": int(np.sum(tl < t64)),
            "fallbacks": int(sum(r["learned"]["fallback"] for r in rows)),
            "max_rel_err_vs_fp64": float(max(r["rel_err_vs_fp64"] for r in rows))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--problems", type=int, default=4000)
    ap.add_argument("--heldout", type=int, default=200)
    ap.add_argument("--heldout-dims", type=int, nargs=3, default=None)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--time-limit", type=float, default=1e9, help="stop labelling after this many seconds")
    ap.add_argument("--dataset", default=None, help="train on this dataset instead of labelling")
    ap.add_argument("--out", required=True)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    import torch

    import amgt_b200
    from amgt_b200 import policy

    amgt_b200.init()
    torch.cuda.set_device(0)
    report = {}
    if args.dataset:
        d = np.load(args.dataset, allow_pickle=False)
        X, T = d["X"], d["T"]
        report["dataset"] = args.dataset
    else:
        t0 = time.perf_counter()
        Xs, Ts, meta = [], [], []
        for k in range(args.problems):
            r = policy.label_problem(k)
            if r is not None:
                Xs.append(r[0])
                Ts.append(r[1])
                meta.append(r[2])
            if time.perf_counter() - t0 > args.time_limit:
                break
        X, T = np.concatenate(Xs), np.concatenate(Ts)
        lab = np.array([[m["seed"], m["theta"], m["class"], m["iters"], m["eps"], m["angle"]] for m in meta])
        np.savez_compressed(os.path.join(args.out, "policy_dataset.npz"), X=X, T=T, labels=lab)
        report["labelling_s"] = round(time.perf_counter() - t0, 1)
        report["problems_labelled"] = len(meta)
        report["theta_star_counts"] = {str(t): int(np.sum(lab[:, 1] == t)) for t in policy.THETAS}
        report["class_counts"] = {str(c): int(np.sum(lab[:, 2] == c)) for c in (0, 1, 2)}
    report["samples"] = int(X.shape[0])
    t0 = time.perf_counter()
    w, hist = policy.train(X, T, epochs=args.epochs, batch=256, lr=2e-3, seed=0)
    report["training_s"] = round(time.perf_counter() - t0, 2)
    report["loss_first_last"] = [float(hist[0]), float(hist[-1])]
    np.save(os.path.join(args.out, "policy_mlp.npy"), w.astype(np.float32))
    if args.heldout > 0:
        rows = evaluate(w, [1_000_000 + k for k in range(args.heldout)], args.heldout_dims)
        report["heldout"] = summarize(rows)
        report["heldout_rows"] = rows
    json.dump(report, open(os.path.join(args.out, "policy_report.json"), "w"), indent=1)
    print(json.dumps({k: v for k, v in report.items() if k != "heldout_rows"}), flush=True)


if __name__ == "__main__":
    main()
