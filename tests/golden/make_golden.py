"""Regenerates the golden fixtures of this directory from the AmgT
repository (read-only).  Run in a checkout where the reference tree is
available:  python tests/golden/make_golden.py /path/to/AmgT

Writes
  hypre_spgemm_known_answers.json
      every ij_mm run of AmgT_HYPRE/src/test/TEST_bench/benchmark_spgemm.jobs
      whose product does not depend on random coarsening (A^2, A^T*A,
      Diag(A)*A on HYPRE's Laplacian generators), with the structural nnz of
      the product HYPRE recorded in benchmark_spgemm.saved.lassen.
  poisson_10x10x10_np1_A.npz
      the 7-point 10x10x10 operator HYPRE printed in binary IJ form
      (AmgT_HYPRE/src/test/TEST_ij/data/poisson_10x10x10_np1/IJ.A.i4f8.*):
      COO rows / cols / values in file order, plus b and x0.
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_jobs(path: str):
    jobs = []
    for line in open(path):
        line = line.strip()
        if not line.startswith("mpirun"):
            continue
        m = re.search(r"> benchmark_spgemm\.out\.(\d+)", line)
        idx = int(m.group(1))
        n = [int(v) for v in re.search(r"-n (\d+) (\d+) (\d+)", line).groups()]
        stencil = "27pt" if "-27pt" in line else "9pt" if "-9pt" in line else ("7pt" if n[2] > 1 else "5pt")
        job = re.search(r"-job (\d+)", line)
        jobs.append({"out": idx, "n": n, "stencil": stencil, "job": int(job.group(1)) if job else 1,
                     "np": int(re.search(r"-np (\d+)", line).group(1)), "cmd": line})
    return jobs


def parse_saved(path: str):
    res = {}
    cur = None
    for line in open(path):
        m = re.match(r"# Output file: benchmark_spgemm\.out\.(\d+)", line)
        if m:
            cur = int(m.group(1))
            continue
        m = re.match(r"(A\^2|A\^T\*A|Diag\(A\)\*A|AH): (\d+) x (\d+), nnz \[CPU (\d+), GPU (\d+)\]", line)
        if m and cur is not None:
            res[cur] = {"product": m.group(1), "rows": int(m.group(2)), "cols": int(m.group(3)),
                        "nnz_cpu": int(m.group(4)), "nnz_gpu": int(m.group(5))}
    return res


def main(ref_root: str) -> None:
    bench = os.path.join(ref_root, "AmgT_HYPRE/src/test/TEST_bench")
    jobs = parse_jobs(os.path.join(bench, "benchmark_spgemm.jobs"))
    saved = parse_saved(os.path.join(bench, "benchmark_spgemm.saved.lassen"))
    cases = []
    for j in jobs:
        s = saved.get(j["out"])
        if s is None or s["product"] == "AH":  # P^T A P depends on random coarsening
            continue
        cases.append({**j, **s})
    with open(os.path.join(HERE, "hypre_spgemm_known_answers.json"), "w") as f:
        json.dump({"source": "AmgT_HYPRE/src/test/TEST_bench/benchmark_spgemm.{jobs,saved.lassen}",
                   "note": "ij_mm -n nx ny nz: default Laplacian (7pt, or 5pt when nz == 1), -9pt, -27pt; "
                           "job 1 = A*A, job 2 = A^T*A, job 5 = Diag(A)*A",
                   "cases": cases}, f, indent=1)

    data = os.path.join(ref_root, "AmgT_HYPRE/src/test/TEST_ij/data/poisson_10x10x10_np1")
    raw = open(os.path.join(data, "IJ.A.i4f8.00000.bin"), "rb").read()
    hdr = np.frombuffer(raw, np.uint64, count=11)
    nnz = int(hdr[6])
    body = raw[88:]
    rows = np.frombuffer(body, np.uint32, count=nnz).astype(np.int32)
    cols = np.frombuffer(body, np.uint32, count=nnz, offset=4 * nnz).astype(np.int32)
    vals = np.frombuffer(body, np.float64, count=nnz, offset=8 * nnz).copy()

    def vec(name):
        r = open(os.path.join(data, name), "rb").read()
        return np.frombuffer(r[64:], np.float64).copy()

    np.savez_compressed(os.path.join(HERE, "poisson_10x10x10_np1_A.npz"), header=hdr.astype(np.int64),
                        rows=rows, cols=cols, vals=vals, b=vec("IJ.b.i4f8.00000.bin"),
                        x0=vec("IJ.x0.i4f8.00000.bin"))
    print(f"{len(cases)} known-answer cases; 10x10x10 operator nnz={nnz}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the AmgT repository checkout>")
    main(sys.argv[1])
