"""Benchmark of the AmgT hot path on B200.

Workload (the GPU-scale configuration): 3D 7-point Poisson on 128^3
(2,097,152 rows, 14,581,760 nonzeros), mBSR 4x4 fp64 (3,620,864 blocks),
seeded uniform x.  One step = one SpMV y = A*x on the finest level, the
operation that drives smoothing and residuals in solve.  The run also
builds the Galerkin hierarchy (A_{l+1} = P^T (A_l P), linear interpolation
P, mBSR SpGEMM) and reports per level the A P, P^T and R (A P) times (best
of three calls, after a warm-up build) and SpMV GB/s; then AMG-PCG setup +
solve to 1e-8 in fp64 and in the mixed form, on this operator and on the
27-point variable-coefficient 96^3 operator (the mixed-precision
configuration).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl amgt|reference]
Under torchrun (N > 1) every rank runs the same workload on its own GPU
(replicas: the path does not shard on one node here); rank 0 prints one
JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "setup+solve s to rtol 1e-8, mixed/learned vs FP64 on 1 B200; SpMV HBM GB/s"
GRID = (128, 128, 128)  # the workload; --grid changes it only for profiling captures
PROFILE_JSON = os.path.join(ROOT, "profiles", "spmv_fp64_7pt128.json")


def spmv_bytes(nblk: int, brow: int, m: int, n: int, val_bytes: int = 8, beta: bool = False) -> int:
    """Algorithmic bytes of one mBSR SpMV: block values + block columns +
    block-row pointers + x + y (+ y read when beta != 0).  The kernel does
    not read the bitmaps (values are zero-padded)."""
    return nblk * (16 * val_bytes + 4) + 4 * (brow + 1) + 8 * n + 8 * m * (2 if beta else 1)


def csr_bytes(nnz: int, m: int, n: int) -> int:
    """Useful bytes of the same product in CSR (values + columns + rowptr + x + y)."""
    return nnz * 12 + 4 * (m + 1) + 8 * n + 8 * m


def max_over_ranks(x: float, device="cpu") -> float:
    """The largest x over all ranks (timings are reported as the max over
    ranks); identity without an initialised process group."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_gbs(bytes_per_rank: int, ms_max: float, world: int) -> float:
    """Aggregate GB/s of `world` replicas that each moved bytes_per_rank in
    ms_max milliseconds (the slowest rank's time)."""
    return world * bytes_per_rank / (ms_max * 1e-3) / 1e9


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_traffic():
    """DRAM read + write bytes per launch of the SpMV from its ncu capture
    (profiles/spmv_fp64_7pt128.json), or None."""
    try:
        return int(json.load(open(PROFILE_JSON))["traffic_bytes_per_launch"])
    except (OSError, KeyError, ValueError):
        return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.proc or not self.out:
            return None
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------- reference
def cpu_spmv_rate(steps: int | None, budget_s: float):
    """CPU SpMV on the same workload, the oracle (C, OpenMP, all host
    threads).  Runs `steps` products, or as many as fit in budget_s."""
    from oracle import oracle as orc

    A = orc.laplacian(*GRID)
    B = orc.csr2bsr(A)
    x = orc.rand_uniform(0, A.n)
    y = np.zeros(A.m)
    orc.lib().orc_bsr_spmv(0, B.m, B.n, B.bptr, B.bidx, B.bval, 1.0, x, 0.0, y)  # warm
    nbytes = spmv_bytes(B.nblk, B.brow, A.m, A.n)
    t0 = time.perf_counter()
    k = 0
    while True:
        orc.lib().orc_bsr_spmv(0, B.m, B.n, B.bptr, B.bidx, B.bval, 1.0, x, 0.0, y)
        k += 1
        el = time.perf_counter() - t0
        if (steps is not None and k >= steps) or (steps is None and el >= budget_s):
            break
    return nbytes * k / el / 1e9, k, el, orc.num_threads()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    steps = max(1, args.steps)
    for _ in range(max(0, args.warmup)):
        cpu_spmv_rate(1, 0)
    gbs, k, el, cores = cpu_spmv_rate(steps, 0)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(gbs, 3), "unit": "GB/s", "n_gpus": args.gpus,
        "steps": k, "warmup": args.warmup, "ms_per_step": round(1e3 * el / k, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"mBSR SpMV y=A*x (fp64), 3D 7-point Poisson {GRID[0]}^3", "parallelism": "host threads"},
        "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": cores, "kind": "port",
                         "sample": f"{k} full SpMVs of the {GRID[0]}^3 operator (C oracle, OpenMP)"},
        "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# -------------------------------------------------------------------- GPU
def spgemm_work(Ah: dict, Bh: dict) -> dict:
    """Work of C = A * B on mBSR (host arrays from Bsr.host()): the (A block,
    B block) pairs, those with a non-zero bitmap product, and the flop counts
    useful = 2 * sum over pairs and k of popc(column k of A's bitmap) *
    popc(row k of B's bitmap), block = 128 per pair with a non-zero product."""
    bptr = Bh["bptr"].astype(np.int64)
    lens = bptr[Ah["bidx"] + 1] - bptr[Ah["bidx"]]
    npairs = int(lens.sum())
    if npairs == 0:
        return {"pairs": 0, "pairs_nonzero": 0, "flops_useful": 0, "flops_block": 0}
    a_of = np.repeat(np.arange(len(lens)), lens)
    first = np.repeat(np.cumsum(lens) - lens, lens)
    b_of = bptr[Ah["bidx"]][a_of] + (np.arange(npairs) - first)
    ma = Ah["bmap"].astype(np.int64)[a_of]
    mb = Bh["bmap"].astype(np.int64)[b_of]
    pc = np.array([bin(i).count("1") for i in range(16)], dtype=np.int64)
    useful = np.zeros(npairs, dtype=np.int64)
    for k in range(4):
        colk = ((ma >> k) & 1) + ((ma >> (k + 4)) & 1) + ((ma >> (k + 8)) & 1) + ((ma >> (k + 12)) & 1)
        useful += colk * pc[(mb >> (4 * k)) & 0xF]
    nz = int(np.count_nonzero(useful))
    return {"pairs": npairs, "pairs_nonzero": nz, "flops_useful": int(2 * useful.sum()), "flops_block": 128 * nz}


def build_hierarchy(amgt, torch, A, grid, max_levels=8, min_rows=512, work=False):
    """Galerkin hierarchy A_{l+1} = P^T (A_l P) with linear interpolation P;
    returns (per-level info, [A_0, A_1, ...]).  work=True adds the products'
    work counts (host copies between levels: the times of that pass are not
    reported)."""
    from amgt_b200 import problems

    levels, mats = [], [A]
    dims = grid
    for lvl in range(max_levels):
        Ab = mats[-1]
        m = Ab.s.row
        info = {"level": lvl, "rows": m, "blocks": Ab.nblk, "nnz": Ab.s.csr_nnz}
        levels.append(info)
        if m <= min_rows or lvl == max_levels - 1:
            break
        (pm, pn, pia, pja, pa), cdims = problems.interp(*dims)
        P = amgt.Bsr.from_csr(pm, pn, torch.from_numpy(pia).cuda(), torch.from_numpy(pja).cuda(),
                              torch.from_numpy(pa).cuda())
        def best_of(fn, reps=3):  # steady state: the first call of a size may grow the memory pool
            best, out = None, None
            for _ in range(reps):
                out = None
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                out = fn()
                torch.cuda.synchronize()
                t = time.perf_counter() - t0
                best = t if best is None else min(best, t)
            return out, best

        (AP, _), t_ap = best_of(lambda: amgt.spgemm(Ab, P, want_csr=False))
        R, t_pt = best_of(P.transpose)
        (RAP, _), t_rap = best_of(lambda: amgt.spgemm(R, AP, want_csr=True))
        info.update({"AP_ms": round(1e3 * t_ap, 3), "PT_ms": round(1e3 * t_pt, 3), "RAP_ms": round(1e3 * t_rap, 3),
                     "P_blocks": P.nblk, "AP_blocks": AP.nblk})
        if work:
            info.update({"AP_work": spgemm_work(Ab.host(), P.host()), "RAP_work": spgemm_work(R.host(), AP.host())})
        del AP, R, P
        mats.append(RAP)
        dims = cdims
    return levels, mats


def geometric_interps(problems, dims, coarse_rows=64):
    """Linear interpolation operators (host CSR) down to <= coarse_rows."""
    Ps = []
    while dims[0] * dims[1] * dims[2] > coarse_rows:
        P, cd = problems.interp(*dims)
        if cd == dims:
            break
        Ps.append(P)
        dims = cd
    return Ps


MIXED_POLICY = [0, 1, 1, 2]  # level 0 fp64, 1-2 fp32, >= 3 fp16 (values); fp32 accumulation
FGMRES_IR = {"solver": 1, "restart": 30, "inner_prec0": 1, "inner_tol": 1e-4}
FGMRES_IR_DESC = ("FGMRES(30) with iterative refinement: fp64 residual and update per refinement step; inner "
                  "FGMRES with level 0 in fp32 (exact fp16 storage where it holds), levels 1-2 fp32, >=3 fp16, "
                  "fp32 Krylov basis, fp64 inner products; Galerkin products at each level's precision")


def amg_setup_solve(amgt, torch, A_host, Ps_host, b_host, policy, smooth0, flexible, reps=3, exact=1, galerkin=0,
                    **extra):
    """Setup + solve to ||b - A x|| / ||b|| <= 1e-8 through the library;
    device-resident inputs.  Returns timings, iterations and the residual
    recomputed in fp64 from the returned x."""
    from amgt_b200.amg import AmgSolver, default_params

    amgt.set_level_policy(policy)
    dev = lambda M: (M[0], M[1]) + tuple(torch.from_numpy(v).cuda() for v in M[2:])  # noqa: E731
    dA, dPs = dev(A_host), [dev(P) for P in Ps_host]
    b = torch.from_numpy(b_host).cuda()
    prm = default_params(flexible=flexible, smooth_prec0=smooth0, exact_storage=exact, galerkin_by_level=galerkin,
                         **extra)
    S = AmgSolver(dA, dPs, prm)  # warm-up: module loads, pools
    S.solve(b)
    S.free()
    torch.cuda.synchronize()
    best = None
    for _ in range(reps):
        t0 = time.perf_counter()
        S = AmgSolver(dA, dPs, prm)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        x, it, rel = S.solve(b)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        run = {"setup_s": t1 - t0, "solve_s": t2 - t1, "iters": it, "relres": rel}
        if best is None or run["setup_s"] + run["solve_s"] < best["setup_s"] + best["solve_s"]:
            best = dict(run, x=x.clone(), levels=[S.level(l) for l in range(S.num_levels())],
                        setup_ms=S.setup_times())
        S.free()
    # fp64 verification of the returned solution (library fp64 SpMV)
    Ab = amgt.Bsr.from_csr(*dA)
    r = b.clone()
    Ab.spmv(best["x"], r, alpha=-1.0, beta=1.0)
    best["relres_fp64_verified"] = float(torch.linalg.vector_norm(r) / torch.linalg.vector_norm(b))
    amgt.set_level_policy([])
    return best


def amg_e2e(amgt, torch, A_host, Ps_host, b_host, policy, smooth0, flexible):
    """Same, end to end from host buffers: CSR + interpolation + b copied to
    the device, setup, solve, x copied back, all inside the timed region."""
    from amgt_b200.amg import AmgSolver, default_params

    amgt.set_level_policy(policy)
    prm = default_params(flexible=flexible, smooth_prec0=smooth0)
    # inputs in pinned host memory (prepared outside the timed region)
    pin = lambda M: (M[0], M[1]) + tuple(torch.from_numpy(v).pin_memory() for v in M[2:])  # noqa: E731
    A_pin, P_pin = pin(A_host), [pin(P) for P in Ps_host]
    b_pin = torch.from_numpy(b_host).pin_memory()
    xh = torch.empty(b_host.shape[0], dtype=torch.float64).pin_memory()
    dev = lambda M: (M[0], M[1]) + tuple(t.cuda(non_blocking=True) for t in M[2:])  # noqa: E731
    samples = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        S = AmgSolver(dev(A_pin), [dev(P) for P in P_pin], prm)
        x, it, rel = S.solve(b_pin.cuda(non_blocking=True))
        xh.copy_(x, non_blocking=True)
        torch.cuda.synchronize()
        samples.append(time.perf_counter() - t0)
        S.free()
        del S, x
    amgt.set_level_policy([])
    h2d = sum(v.nbytes for M in [A_host] + list(Ps_host) for v in M[2:]) + b_host.nbytes
    return {"value": round(sorted(samples)[1], 4), "unit": "s", "statistic": "median of 3 calls",
            "samples_s": [round(t, 4) for t in samples], "iters": it, "h2d_bytes": int(h2d),
            "d2h_bytes": int(xh.numel() * 8)}


def spmm_bytes(nblk: int, brow: int, m: int, n: int, nvec: int, val_bytes: int, beta: bool = False) -> int:
    """Algorithmic bytes of one row-major SpMM: block values + block columns
    + block-row pointers + X once + Y written (+ Y read when beta != 0)."""
    return nblk * (16 * val_bytes + 4) + 4 * (brow + 1) + 8 * n * nvec + 8 * m * nvec * (2 if beta else 1)


def batching_report(amgt, torch, problems, stream):
    """The batching form: (a) 7-point 64^3 with 32 right-hand sides
    (amgt_amg_solve_multi: every cycle operator one SpMM over all columns;
    the 32-vector SpMM timed alone, with the autotuner's choice) against 32
    single-right-hand-side solves; (b) 64 2D 5-point systems with sides
    uniform in [32, 512] (seed 0) in one graph launch (amgt_batch_setup +
    amgt_amg_solve_batch) against 64 solves one after another."""
    from amgt_b200.amg import AmgSolver, BatchSolver, default_params

    out = {}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dims = (64, 64, 64)
    m, n, ia, ja, a = problems.laplacian(*dims)
    dA = (m, n) + tuple(torch.from_numpy(v).cuda() for v in (ia, ja, a))
    Ps = geometric_interps(problems, dims)
    dPs = [(P[0], P[1]) + tuple(torch.from_numpy(v).cuda() for v in P[2:]) for P in Ps]
    nv = 32
    B = torch.from_numpy(np.ascontiguousarray(np.stack([problems.rand_uniform(v, n) for v in range(nv)], axis=1))).cuda()
    # the SpMM alone: fp32-requested values (the exact fp16 shadow) on the tensor cores vs CUDA cores
    G = amgt.Bsr.from_csr(*dA)
    G.make_exact()
    tune = G.autotune(prec=1, nvec=nv)
    X = torch.rand(n, nv, dtype=torch.float64, device="cuda")
    Y = torch.zeros(m, nv, dtype=torch.float64, device="cuda")
    vb = 2 if G.s.exact_prec == 2 else 4
    nbytes = spmm_bytes(G.nblk, G.s.blc_row, m, n, nv, vb)
    spmm = {"workload": f"7-point {dims[0]}^3, {nv} right-hand sides, fp32 values read from the exact fp16 shadow",
            "bytes_per_call": nbytes, "autotune_ms": {str(k): round(v, 5) for k, v in tune["ms"].items()},
            "autotune_choice": tune["choice"], "choice_code": "10 * engine (0 CUDA cores, 1 tensor cores) + warps/CTA"}
    for name, eng in (("tensor_cores", 2), ("cuda_cores", 1), ("autotuned", 0)):
        for _ in range(3):
            G.spmm_rm(X, Y, prec=1, engine=eng)
        ev0.record(stream)
        for _ in range(20):
            G.spmm_rm(X, Y, prec=1, engine=eng)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1) / 20
        spmm[name] = {"ms": round(ms, 5), "gbs": round(nbytes / (ms * 1e-3) / 1e9, 1)}
    peak, _ = read_peaks()
    spmm["roofline"] = {"bound": "hbm", "achieved": spmm["autotuned"]["gbs"], "peak": peak, "unit": "GB/s",
                        "frac": round(spmm["autotuned"]["gbs"] / peak, 4)}
    out["spmm_64cubed_32rhs"] = spmm
    del G, X, Y
    # (a) the multi-right-hand-side solve, mixed: levels 1-2 fp32, >= 3 fp16,
    # level 0 in the correction fp32; fp64 refinement.  Best of three
    # setup + first solve on a new handle (after a warm-up), and a second
    # solve on the same handle (the steady state)
    amgt.set_level_policy(MIXED_POLICY)
    prm = default_params(inner_prec0=1, galerkin_by_level=1)
    S = AmgSolver(dA, dPs, prm)
    S.solve_multi(B)  # warm-up (module loads, pool growth)
    S.free()
    best = None
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        S = AmgSolver(dA, dPs, prm)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        Xs, its, rel = S.solve_multi(B)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        S.solve_multi(B, torch.zeros_like(B))
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        S.free()
        run = (t1 - t0, t2 - t1, t3 - t2)
        if best is None or sum(run[:2]) < sum(best[:2]):
            best = run
    amgt.set_level_policy([])
    multi = {"setup_s": round(best[0], 5), "solve_s": round(best[1], 5), "second_solve_s": round(best[2], 5),
             "iters_per_column": [min(its), max(its)], "max_rel_res": max(rel),
             "statistic": "best of 3 (setup + first solve on a new handle); second_solve_s: same handle again"}
    # the same 32 right-hand sides one at a time (plain fp64 PCG, one graph launch each)
    amgt.set_level_policy([0])
    S = AmgSolver(dA, dPs, default_params())
    b0 = B[:, 0].contiguous()
    S.solve(b0)
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    for v in range(nv):
        S.solve(B[:, v].contiguous())
    torch.cuda.synchronize()
    t4 = time.perf_counter()
    S.free()
    amgt.set_level_policy([])
    multi["one_at_a_time_fp64_solve_s"] = round(t4 - t3, 5)
    multi["speedup_solve"] = round((t4 - t3) / multi["solve_s"], 2)
    multi["speedup_second_solve"] = round((t4 - t3) / multi["second_solve_s"], 2)
    out["multi_rhs_64cubed_32"] = multi
    # (b) 64 uneven systems in one launch
    sides = np.random.default_rng(0).integers(32, 513, size=64)
    systems = []
    for side in sides:
        sm, sn, sia, sja, sa = problems.laplacian(int(side), int(side), 1)
        sA = (sm, sn) + tuple(torch.from_numpy(v).cuda() for v in (sia, sja, sa))
        sPs = [(P[0], P[1]) + tuple(torch.from_numpy(v).cuda() for v in P[2:])
               for P in geometric_interps(problems, (int(side), int(side), 1))]
        systems.append((sA, sPs))
    rows = sum(int(s_) ** 2 for s_ in sides)
    bb = torch.from_numpy(np.concatenate([problems.rand_uniform(i, int(s_) ** 2) for i, s_ in enumerate(sides)])).cuda()
    amgt.set_level_policy([0])
    Bs = BatchSolver(systems)
    Bs.solve_batch(bb)  # warm-up
    Bs.free()
    best = None
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Bs = BatchSolver(systems)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        xb, its, rel, loop_it = Bs.solve_batch(bb)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        off = Bs.offsets
        Bs.free()
        if best is None or t2 - t0 < best[2] - best[0]:
            best = (t0, t1, t2)
    t0, t1, t2 = best
    # one system at a time
    t3 = time.perf_counter()
    for i, (sA, sPs) in enumerate(systems):
        S = AmgSolver(sA, sPs)
        S.solve(bb[off[i]:off[i + 1]].contiguous())
        S.free()
    torch.cuda.synchronize()
    t4 = time.perf_counter()
    amgt.set_level_policy([])
    out["batch_64_systems"] = {
        "systems": 64, "sides": [int(min(sides)), int(max(sides))], "rows": rows, "setup_s": round(t1 - t0, 5),
        "solve_s": round(t2 - t1, 5), "total_s": round(t2 - t0, 5), "loop_iterations": loop_it,
        "iters_per_system": [min(its), max(its)], "max_rel_res": max(rel),
        "one_system_at_a_time_total_s": round(t4 - t3, 5), "speedup_total": round((t4 - t3) / (t2 - t0), 2),
        "statistic": "best of 3 (setup + solve on a new handle, after a warm-up); the baseline: one pass over the "
                     "64 systems, a new handle per system",
        "solve_launches": "one CUDA graph launch (a conditional while node) for every iteration of every system"}
    return out


def learned_report(n_seeds: int):
    """The learned precision / theta policy (amgt_b200/data/policy_mlp.npy)
    against the plain FP64 configuration (theta 0.25, every level fp64) on
    held-out rotated anisotropic 128^3 problems (seeds 1,000,000 + k): setup
    (level by level through the coarsening callback) + solve to 1e-8, the
    convergence factor as the yardstick; a learned solve that misses 1e-8 falls
    back to fp64 and is charged both runs."""
    from amgt_b200 import policy
    from amgt_b200.train_policy import evaluate, summarize

    w = np.load(policy.WEIGHTS)
    rows = evaluate(w, [1_000_000 + k for k in range(n_seeds)])
    out = summarize(rows)
    out["problems_desc"] = ("rotated anisotropic diffusion 128^3 (2,097,152 rows), eps log-uniform in [1e-3, 1], "
                            "angle uniform in [0, pi), b uniform[-1,1]; seeds 1,000,000..")
    out["training"] = "4,000 seeded problems 32^2..64^3 labelled by the plain solver; amgt_b200/data/policy_report.json"
    return out


def boomer_report(amgt, torch, A_host, grid, cpu: bool, problem: str | None = None, recorded: bool = True):
    """The metric's setup + solve on its stated settings: BoomerAMG's HMIS
    (theta 0.25) + ext+i (P_max 4) hierarchy, built on the host as HYPRE's
    CPU setup builds it (amgt_boomer_hierarchy_host), then the GPU's
    Galerkin products, smoothers and PCG (fp64 / mixed / mixed FGMRES-IR).
    b = the ij driver's -rhsrand vector, so the fp64 iterations and final
    residual compare with the reference's recorded CPU BoomerAMG run."""
    import scipy.sparse as sp

    from amgt_b200 import boomer

    m, n, ia, ja, a = A_host
    t0 = time.perf_counter()
    Ps, As = boomer.hypre_hierarchy(sp.csr_matrix((a, ja, ia), shape=(m, n)))
    for P in Ps:  # same operator; sorted rows take the conversion's merge path
        P.sort_indices()
    host_s = time.perf_counter() - t0
    Ps_host = [(P.shape[0], P.shape[1], P.indptr.astype(np.int32), P.indices.astype(np.int32), P.data) for P in Ps]
    b_host = boomer.ij_random_rhs(m)
    f64 = amg_setup_solve(amgt, torch, A_host, Ps_host, b_host, [0], 0, 0)
    mix = amg_setup_solve(amgt, torch, A_host, Ps_host, b_host, MIXED_POLICY, 1, 1, galerkin=1)
    gir = amg_setup_solve(amgt, torch, A_host, Ps_host, b_host, MIXED_POLICY, 1, 0, galerkin=1, **FGMRES_IR)
    amgt.lib().amgt_spgemm_set_engine(2)  # fp16 Galerkin products of levels >= 3 on the tensor cores
    try:
        mtc = amg_setup_solve(amgt, torch, A_host, Ps_host, b_host, MIXED_POLICY, 1, 1, galerkin=1)
    finally:
        amgt.lib().amgt_spgemm_set_engine(0)
    dev_levels = None
    if recorded:
        # the same settings level by level from the GPU's own products
        # (amgt_boomer_interp in the coarsening callback: each A_l copied to
        # the host, sorted, coarsened there; P_l uploaded)
        dA = (m, n) + tuple(torch.from_numpy(np.ascontiguousarray(v)).cuda() for v in (ia, ja, a))
        b = torch.from_numpy(b_host).cuda()
        amgt.set_level_policy([0])
        try:
            runs = []
            for _ in range(2):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                S = boomer.BoomerSolver(dA, levels="device")
                torch.cuda.synchronize()
                t1 = time.perf_counter()
                x, it, rel = S.solve(b)
                torch.cuda.synchronize()
                t2 = time.perf_counter()
                runs.append({"setup_s": round(t1 - t0, 4), "solve_s": round(t2 - t1, 5), "iters": it,
                             "relres": float(f"{rel:.7g}"),
                             "levels": [S.level(l)["rows"] for l in range(S.num_levels())],
                             "operator_complexity": round(S.operator_complexity(), 4)})
                S.free()
        finally:
            amgt.set_level_policy([])
        dev_levels = dict(runs[-1], what="fp64, coarsening from the GPU's Galerkin products level by level "
                                         "(host HMIS + ext+i on each sorted A_l, P_l uploaded); setup includes "
                                         "that host work; second of two runs")
    nnz = [int(M.nnz) for M in As]
    rep = {"problem": (problem or f"3D 7-point Poisson {grid[0]}^3") + ", b = ij -rhsrand (seed 22775, unit norm), "
                      "BoomerAMG settings: HMIS theta 0.25, ext+i P_max 4, l1-Jacobi V(1,1), tol 1e-8",
           "levels": [int(M.shape[0]) for M in As], "operator_complexity": round(sum(nnz) / nnz[0], 4),
           "host_coarsening_s": round(host_s, 3),
           "host_coarsening": "HMIS + ext+i + truncation + HYPRE-order Galerkin products on the host, one "
                              "thread (HYPRE 2.31 runs HMIS on the host in GPU builds too); the same P for "
                              "every form below",
           }
    if dev_levels is not None:
        rep["fp64_device_levels"] = dev_levels
    if recorded:
        rep["reference_recorded"] = {"iters": 11, "relres": 2.411373e-09, "levels": 9, "operator_complexity": 3.27,
                                     "what": "HYPRE 2.31 CPU BoomerAMG from the AmgT tree, ij -rhsrand"}
    for name, rres in (("fp64", f64), ("mixed", mix), ("mixed_fgmres_ir", gir), ("mixed_tensor_core_products", mtc)):
        rep[name] = {k: float(f"{rres[k]:.7g}") if isinstance(rres[k], float) else rres[k]
                     for k in ("setup_s", "solve_s", "iters", "relres", "relres_fp64_verified")}
        rep[name]["total_s"] = round(rres["setup_s"] + rres["solve_s"], 5)
        rep[name]["setup_ms"] = {k: round(v, 3) for k, v in rres["setup_ms"].items()}
    for name, rres in (("mixed", mix), ("mixed_fgmres_ir", gir), ("mixed_tensor_core_products", mtc)):
        rep[name]["speedup_vs_fp64"] = round(rep["fp64"]["total_s"] / rep[name]["total_s"], 3)
        rep[name]["rel_err_vs_fp64_solution"] = float(
            torch.linalg.vector_norm(rres["x"] - f64["x"]) / torch.linalg.vector_norm(f64["x"]))
    rep["mixed"]["policy"] = "levels 0 fp64 (residual) / fp32 smoother, 1-2 fp32, >=3 fp16; flexible CG"
    rep["mixed_fgmres_ir"]["policy"] = FGMRES_IR_DESC
    rep["mixed_tensor_core_products"]["policy"] = ("as mixed, with the fp16 Galerkin products (levels >= 3) on the "
                                                   "tensor cores (amgt_spgemm_set_engine, mma.m16n8k16)")
    if cpu:
        from oracle import oracle as orc

        Pc = []
        for P in Ps:
            P = P.copy()
            P.sort_indices()
            Pc.append(orc.CSR(P.shape[0], P.shape[1], P.indptr.astype(np.int32), P.indices.astype(np.int32),
                              P.data))
        A = orc.CSR(m, n, ia, ja, a)
        t0 = time.perf_counter()
        h = orc.Amg(A, Pc)
        t1 = time.perf_counter()
        xo, it, rel, _ = h.solve(b_host)
        t2 = time.perf_counter()
        rep["cpu_oracle"] = {"setup_s": round(t1 - t0 + host_s, 3), "solve_s": round(t2 - t1, 3),
                             "total_s": round(t2 - t0 + host_s, 3), "iters": it, "relres": float(f"{rel:.7g}"),
                             "cores": orc.num_threads(), "kind": "port",
                             "what": "the oracle's AMG-PCG (C, OpenMP) on the same BoomerAMG hierarchy; setup "
                                     "includes the host coarsening above"}
        rep["fp64"]["rel_err_vs_cpu_oracle"] = float(np.linalg.norm(f64["x"].cpu().numpy() - xo) / np.linalg.norm(xo))
    return rep


def boomer_setup_only(grid, mixed: bool = False, engine: int = 0, operator: str = "7pt", solves: int = 0,
                      packed: int = 0):
    """Profiling captures: the BoomerAMG hierarchy of the 7-point operator
    built on the host, then two setups on the GPU (the first loads the
    modules), fp64 or the mixed policy with Galerkin products at each
    level's precision on the given SpGEMM engine; prints the second one's
    phase times, then (solves > 0) that many solves of the ij driver's
    right-hand side on the second setup, with the last one's time."""
    import scipy.sparse as sp
    import torch

    import amgt_b200 as amgt
    from amgt_b200 import boomer, problems
    from amgt_b200.amg import AmgSolver, default_params

    m, n, ia, ja, a = problems.laplacian(*grid) if operator == "7pt" else problems.varcoef27(*grid, seed=1)
    Ps, _ = boomer.hypre_hierarchy(sp.csr_matrix((a, ja, ia), shape=(m, n)))
    dev = lambda *v: tuple(torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in v)  # noqa: E731
    dPs = []
    for P in Ps:
        P.sort_indices()
        dPs.append((P.shape[0], P.shape[1]) + dev(P.indptr.astype(np.int32), P.indices.astype(np.int32), P.data))
    dA = (m, n) + dev(ia, ja, a)
    amgt.set_level_policy(MIXED_POLICY if mixed else [0])
    amgt.lib().amgt_spgemm_set_engine(engine)
    prm = default_params(flexible=1, smooth_prec0=1, galerkin_by_level=1) if mixed else default_params()
    prm.packed = packed
    for rep in range(2):
        S = AmgSolver(dA, dPs, prm)
        torch.cuda.synchronize()
        times = S.setup_times()
        if rep == 0:
            S.free()
    amgt.lib().amgt_spgemm_set_engine(0)
    amgt.set_level_policy([])
    print(json.dumps({"boomer_setup_ms": {k: round(v, 3) for k, v in times.items()}}))
    if solves > 0:
        b = torch.from_numpy(boomer.ij_random_rhs(m)).cuda()
        for _ in range(solves):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _, it, rel = S.solve(b)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
        print(json.dumps({"boomer_solve_ms": round(1e3 * (t1 - t0), 3), "iters": it, "relres": rel}))
    S.free()


def cpu_amg(grid, b_host):
    """The oracle's AMG-PCG (C, OpenMP, all host threads) on the same problem."""
    from oracle import oracle as orc

    A = orc.laplacian(*grid)
    Ps = orc.geometric_hierarchy(*grid)
    t0 = time.perf_counter()
    h = orc.Amg(A, Ps)
    t1 = time.perf_counter()
    x, it, rel, _ = h.solve(b_host)
    t2 = time.perf_counter()
    return {"setup_s": round(t1 - t0, 3), "solve_s": round(t2 - t1, 3), "total_s": round(t2 - t0, 3), "iters": it,
            "relres": rel, "cores": orc.num_threads(), "kind": "port"}, x


def run_amgt(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    import amgt_b200 as amgt
    from amgt_b200 import problems

    amgt.init()
    m, n, ia, ja, a = problems.laplacian(*GRID)
    x_host = problems.rand_uniform(0, n)
    ia_d, ja_d, a_d = (torch.from_numpy(v).cuda() for v in (ia, ja, a))
    A = amgt.Bsr.from_csr(m, n, ia_d, ja_d, a_d)
    x = torch.from_numpy(x_host).cuda()
    y = torch.zeros(m, dtype=torch.float64, device="cuda")
    nbytes = spmv_bytes(A.nblk, A.s.blc_row, m, n)
    ubytes = csr_bytes(int(ja.size), m, n)

    # warm-up (untimed)
    for _ in range(max(3, args.warmup)):
        A.spmv(x, y)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = amgt.kernel_launch_count()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            A.spmv(x, y)
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = amgt.kernel_launch_count() - launches0
    ms = ev0.elapsed_time(ev1) / args.steps
    ms_max = max_over_ranks(ms, device="cuda")
    if world > 1:
        dist.barrier()
    value = whole_job_gbs(nbytes, ms_max, world)
    per_gpu = nbytes / (ms * 1e-3) / 1e9

    # the same product on the bitmap-packed values (what the solver runs)
    Apk = A.pack(0)
    pbytes = A.nblk * 10 + 8 * Apk.s.nnz + 4 * (A.s.blc_row + 1) + 8 * n + 8 * m
    for _ in range(3):
        Apk.spmv(x, y)
    ev0.record(stream)
    for _ in range(args.steps):
        Apk.spmv(x, y)
    ev1.record(stream)
    torch.cuda.synchronize()
    pms = ev0.elapsed_time(ev1) / args.steps
    packed = {"ms_per_step": round(pms, 5), "bytes_per_step": pbytes,
              "achieved_gbs": round(pbytes / (pms * 1e-3) / 1e9, 2),
              "csr_useful_gbs": round(ubytes / (pms * 1e-3) / 1e9, 2),
              "speedup_vs_16_value_blocks": round(ms / pms, 3)}
    del Apk

    # e2e: host x in, host y out, through the C ABI, every step.  Serial:
    # upload, product, download on one stream.  Pipelined: steps rotate over
    # three streams with their own x / y, so one step's y download (device ->
    # host) and the product run while the next step's x upload (host ->
    # device) does, and an upload never waits for its stream's previous
    # download; every step still moves its full x and y across PCIe.
    NS = 3
    xh = torch.from_numpy(x_host).pin_memory()
    yhs = [torch.empty(m, dtype=torch.float64).pin_memory() for _ in range(NS)]
    xs = [x] + [torch.empty_like(x) for _ in range(NS - 1)]
    ys = [y] + [torch.empty_like(y) for _ in range(NS - 1)]
    streams = [stream] + [torch.cuda.Stream() for _ in range(NS - 1)]

    def e2e_step(i, pipelined):
        j = i % NS if pipelined else 0
        with torch.cuda.stream(streams[j]):
            xs[j].copy_(xh, non_blocking=True)
            A.spmv(xs[j], ys[j])
            yhs[j].copy_(ys[j], non_blocking=True)

    def e2e_time(pipelined):
        for i in range(NS):
            e2e_step(i, pipelined)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ev0.record(stream)
        for sj in streams[1:]:
            sj.wait_event(ev0)
        for i in range(args.steps):
            e2e_step(i, pipelined)
        for sj in streams[1:]:
            stream.wait_stream(sj)
        ev1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(ev0.elapsed_time(ev1) / args.steps, device="cuda")

    e2e_serial_ms = e2e_time(False)
    e2e_ms = e2e_time(True)
    e2e_value = whole_job_gbs(nbytes, e2e_ms, world)
    e2e_serial = whole_job_gbs(nbytes, e2e_serial_ms, world)
    if not all(torch.equal(yhs[0], yh) for yh in yhs[1:]):
        raise RuntimeError("pipelined e2e steps disagree")

    # hierarchy: RAP per level and SpMV GB/s per level (not part of `value`);
    # built twice, the first pass loading the kernels' modules
    levels, mats = [], []
    if not args.no_levels:
        build_hierarchy(amgt, torch, A, GRID)  # warm-up pass, result dropped
        levels, mats = build_hierarchy(amgt, torch, A, GRID)
        # work per product (pairs, flops) from a third, untimed pass
        counted, _ = build_hierarchy(amgt, torch, A, GRID, work=True)
        for info, c in zip(levels, counted):
            for key, t in (("AP_work", info.get("AP_ms")), ("RAP_work", info.get("RAP_ms"))):
                if key in c:
                    info[key] = c[key]
                    info[key[:-5] + "_gflops_block"] = round(c[key]["flops_block"] / (t * 1e-3) / 1e9, 1)
    for lvl, Ab in enumerate(mats):
        xx = torch.zeros(Ab.s.col, dtype=torch.float64, device="cuda").uniform_(-1, 1)
        yy = torch.zeros(Ab.s.row, dtype=torch.float64, device="cuda")
        Pk = Ab.pack(0)
        for op, name, nb in ((Ab.spmv, "spmv", spmv_bytes(Ab.nblk, Ab.s.blc_row, Ab.s.row, Ab.s.col)),
                             (Pk.spmv, "packed_spmv", Ab.nblk * 10 + 8 * Pk.s.nnz + 4 * (Ab.s.blc_row + 1)
                              + 8 * (Ab.s.row + Ab.s.col))):
            for _ in range(3):
                op(xx, yy)
            reps = 20
            ev0.record(stream)
            for _ in range(reps):
                op(xx, yy)
            ev1.record(stream)
            torch.cuda.synchronize()
            lms = ev0.elapsed_time(ev1) / reps
            levels[lvl][name + "_ms"] = round(lms, 4)
            levels[lvl][name + "_gbs"] = round(nb / (lms * 1e-3) / 1e9, 1)
        del Pk
    del mats

    # setup + solve to 1e-8: plain fp64 and mixed precision (the metric's first part)
    setup_solve = None
    if not args.no_solve:
        Ps_host = geometric_interps(problems, GRID)
        A_host = (m, n, ia, ja, a)
        b_host = problems.rand_uniform(0, n)
        f64 = amg_setup_solve(amgt, torch, A_host, Ps_host, b_host, [0], 0, 0)
        f64_8 = amg_setup_solve(amgt, torch, A_host, Ps_host, b_host, [0], 0, 0, exact=0)
        mix = amg_setup_solve(amgt, torch, A_host, Ps_host, b_host, MIXED_POLICY, 1, 1, galerkin=1)
        gir = amg_setup_solve(amgt, torch, A_host, Ps_host, b_host, MIXED_POLICY, 1, 0, galerkin=1,
                              **FGMRES_IR)
        err = float(torch.linalg.vector_norm(mix["x"] - f64["x"]) / torch.linalg.vector_norm(f64["x"]))
        setup_solve = {}
        for name, rres in (("fp64", f64), ("fp64_8byte_values", f64_8), ("mixed", mix),
                           ("mixed_fgmres_ir", gir)):
            setup_solve[name] = {k: (float(f"{v:.5g}") if isinstance(v, float) else v) for k, v in rres.items()
                                 if k not in ("x", "levels", "setup_ms")}
            setup_solve[name]["total_s"] = round(rres["setup_s"] + rres["solve_s"], 5)
            setup_solve[name]["setup_ms"] = {k: round(v, 3) for k, v in rres["setup_ms"].items()}
            setup_solve[name]["levels"] = rres["levels"]
        setup_solve["fp64"]["storage"] = ("operators whose values fp16 / fp32 hold exactly read from that shadow "
                                          "(exact_storage=1, the default)")
        setup_solve["fp64_8byte_values"]["storage"] = "exact_storage=0: every operator read as 8-byte values"
        setup_solve["fp64_8byte_values"]["x_bit_identical_to_fp64"] = bool(
            torch.equal(f64["x"].view(torch.int64), f64_8["x"].view(torch.int64)))
        setup_solve["mixed"]["policy"] = ("levels 0 fp64 (residual) / fp32 smoother, 1-2 fp32, >=3 fp16; Galerkin "
                                          "products at each level's precision; flexible CG")
        setup_solve["mixed"]["rel_err_vs_fp64_solution"] = err
        setup_solve["mixed"]["speedup_vs_fp64"] = round(setup_solve["fp64"]["total_s"] / setup_solve["mixed"]["total_s"], 3)
        setup_solve["mixed_fgmres_ir"]["policy"] = FGMRES_IR_DESC
        setup_solve["mixed_fgmres_ir"]["rel_err_vs_fp64_solution"] = float(
            torch.linalg.vector_norm(gir["x"] - f64["x"]) / torch.linalg.vector_norm(f64["x"]))
        setup_solve["mixed_fgmres_ir"]["speedup_vs_fp64"] = round(
            setup_solve["fp64"]["total_s"] / setup_solve["mixed_fgmres_ir"]["total_s"], 3)
        setup_solve["e2e_fp64"] = amg_e2e(amgt, torch, A_host, Ps_host, b_host, [0], 0, 0)
        setup_solve["problem"] = (f"3D 7-point Poisson {GRID[0]}^3, b uniform[-1,1] seed 0, linear-interpolation "
                                  f"hierarchy ({len(Ps_host) + 1} levels), PCG + V(1,1) l1-Jacobi, tol 1e-8")
        # the mixed-precision configuration: 27-point variable-coefficient
        # diffusion 96^3 (log-normal cell coefficients, seed 1), whose values
        # no narrow format holds exactly
        vdims = (96, 96, 96)
        V_host = problems.varcoef27(*vdims, seed=1)
        VPs_host = geometric_interps(problems, vdims)
        vb_host = problems.rand_uniform(0, V_host[0])
        vf64 = amg_setup_solve(amgt, torch, V_host, VPs_host, vb_host, [0], 0, 0)
        vmix = amg_setup_solve(amgt, torch, V_host, VPs_host, vb_host, MIXED_POLICY, 1, 1, galerkin=1)
        vgir = amg_setup_solve(amgt, torch, V_host, VPs_host, vb_host, MIXED_POLICY, 1, 0, galerkin=1, **FGMRES_IR)
        vc = {"problem": "3D 27-point variable-coefficient diffusion 96^3 (884,736 rows, 23.4 M nonzeros), "
                         "b uniform[-1,1] seed 0, linear-interpolation hierarchy, PCG + V(1,1) l1-Jacobi, tol 1e-8"}
        for name, rres in (("fp64", vf64), ("mixed", vmix), ("mixed_fgmres_ir", vgir)):
            vc[name] = {k: float(f"{rres[k]:.5g}") if isinstance(rres[k], float) else rres[k]
                        for k in ("setup_s", "solve_s", "iters", "relres_fp64_verified")}
            vc[name]["total_s"] = round(rres["setup_s"] + rres["solve_s"], 5)
            vc[name]["setup_ms"] = {k: round(v, 3) for k, v in rres["setup_ms"].items()}
        for name, rres in (("mixed", vmix), ("mixed_fgmres_ir", vgir)):
            vc[name]["speedup_vs_fp64"] = round(vc["fp64"]["total_s"] / vc[name]["total_s"], 3)
            vc[name]["rel_err_vs_fp64_solution"] = float(
                torch.linalg.vector_norm(rres["x"] - vf64["x"]) / torch.linalg.vector_norm(vf64["x"]))
        vc["mixed_fgmres_ir"]["policy"] = FGMRES_IR_DESC
        setup_solve["varcoef27_96"] = vc
        setup_solve["boomeramg_128"] = boomer_report(amgt, torch, A_host, GRID,
                                                     cpu=world == 1 and rank == 0 and not args.no_cpu)
        # config 3's operator with the same settings (no recorded reference run)
        setup_solve["boomeramg_varcoef27_96"] = boomer_report(
            amgt, torch, V_host, vdims, cpu=False, recorded=False,
            problem="3D 27-point variable-coefficient diffusion 96^3 (884,736 rows, 23.4 M nonzeros)")
        if world == 1 and rank == 0 and not args.no_cpu:
            setup_solve["cpu_oracle"], xo = cpu_amg(GRID, b_host)
            setup_solve["fp64"]["rel_err_vs_cpu_oracle"] = float(
                np.linalg.norm(f64["x"].cpu().numpy() - xo) / np.linalg.norm(xo))

    batching = None
    if not args.no_batch:
        batching = batching_report(amgt, torch, problems, stream)
    learned = None
    if not args.no_learned and world == 1:
        learned = learned_report(args.learned_seeds)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    peak, peak_kind = read_peaks()
    cpu = None
    if world == 1 and not args.no_cpu:
        gbs, k, el, cores = cpu_spmv_rate(None, args.cpu_seconds)
        cpu = {"value": round(gbs, 3), "unit": "GB/s", "cores": cores, "kind": "port",
               "sample": f"{k} full SpMVs of the 128^3 operator in {el:.1f} s (C oracle, OpenMP)"}
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": round(ms_max, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"mBSR SpMV y=A*x (fp64), 3D 7-point Poisson {GRID[0]}^3: {m:,} rows, "
                               f"{int(ja.size):,} nnz, {A.nblk:,} 4x4 blocks", "global_batch": world,
                   "bytes_per_step": nbytes, "l2": "inputs larger than L2 (matrix 478 MB > 126 MB)",
                   "parallelism": f"replicas{world}"},
        "spmv_useful_gbs": round(world * ubytes / (ms_max * 1e-3) / 1e9, 2),
        "packed_spmv": packed,
        "roofline": {"bound": "hbm", "achieved": round(per_gpu, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(per_gpu / peak, 4), "traffic": read_traffic(),
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                     else "fallback"},
        "cpu_baseline": cpu,
        "e2e": {"value": round(e2e_value, 2), "unit": "GB/s", "h2d_bytes_per_step": 8 * n,
                "d2h_bytes_per_step": 8 * m, "pipelined": "three streams: step k's y download and product overlap "
                "step k+1's x upload", "serial_value": round(e2e_serial, 2)},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "levels": levels,
        "setup_solve": setup_solve,
        "batching": batching,
        "learned_policy": learned,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["amgt", "reference"], default="amgt")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-levels", action="store_true", help="skip the hierarchy / per-level report")
    ap.add_argument("--no-solve", action="store_true", help="skip the AMG setup + solve report")
    ap.add_argument("--no-batch", action="store_true", help="skip the batching-form report")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-policy report")
    ap.add_argument("--learned-seeds", type=int, default=20, help="held-out 128^3 problems in that report")
    ap.add_argument("--grid", type=int, default=128, help="cube side (profiling captures only)")
    ap.add_argument("--boomer-setup-only", action="store_true",
                    help="profiling captures only: one fp64 AMG setup on the BoomerAMG hierarchy of the --grid "
                         "7-point operator (after one warm-up setup), no JSON line")
    ap.add_argument("--setup-mixed", action="store_true", help="with --boomer-setup-only: the mixed policy")
    ap.add_argument("--operator", choices=["7pt", "27pt-varcoef"], default="7pt",
                    help="with --boomer-setup-only: the 7-point operator or the 27-point variable-coefficient one")
    ap.add_argument("--boomer-solves", type=int, default=0,
                    help="with --boomer-setup-only: that many solves after the setup (the last one timed)")
    ap.add_argument("--packed", type=int, default=0,
                    help="with --boomer-setup-only: amgt_amg_params.packed (1: bitmap-packed values in the cycle)")
    ap.add_argument("--spgemm-engine", type=int, default=0,
                    help="with --boomer-setup-only: amgt_spgemm_set_engine (2: fp16 / bf16 products on the tensor "
                         "cores)")
    args = ap.parse_args()
    global GRID
    GRID = (args.grid, args.grid, args.grid)
    if args.boomer_setup_only:
        boomer_setup_only(GRID, args.setup_mixed, args.spgemm_engine, args.operator, args.boomer_solves,
                          args.packed)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_amgt(args)


if __name__ == "__main__":
    main()
