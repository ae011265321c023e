"""CPU tests of bench.py's host logic: the max-over-ranks timing across two
gloo ranks, the whole-job rate, and the CPU reference arm's JSON line."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 1.5 + rank  # the slower rank sets the time
        out[rank] = bench.max_over_ranks(ms)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
        assert dict(out) == {0: 2.5, 1: 2.5}


def test_whole_job_rate_and_single_rank_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.25) == 3.25
    assert bench.whole_job_gbs(500_000_000, 0.1, 1) == pytest.approx(5000.0)
    assert bench.whole_job_gbs(500_000_000, 0.1, 8) == pytest.approx(40000.0)


def test_reference_arm_json_line_on_cpu():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--grid", "24",
                        "--steps", "3", "--warmup", "1"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "GB/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1


def test_reference_arm_rank_nonzero_prints_nothing():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--grid", "16",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=300, cwd=ROOT,
                       env=env)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_spgemm_work_counts_match_brute_force(orc):
    """bench.spgemm_work (pairs, non-zero bitmap products, useful and block
    flops of an mBSR product) against a per-entry count."""
    import bench

    A = orc.varcoef27(9, 8, 7, seed=2)
    P, _ = orc.interp(9, 8, 7)
    BA, BP = orc.csr2bsr(A), orc.csr2bsr(P)
    w = bench.spgemm_work({"bptr": BA.bptr, "bidx": BA.bidx, "bmap": BA.bmap},
                          {"bptr": BP.bptr, "bidx": BP.bidx, "bmap": BP.bmap})
    pairs = nz = useful = 0
    for i in range(BA.brow):
        for p in range(BA.bptr[i], BA.bptr[i + 1]):
            ma, k = int(BA.bmap[p]), BA.bidx[p]
            for q in range(BP.bptr[k], BP.bptr[k + 1]):
                mb = int(BP.bmap[q])
                u = sum(((ma >> (4 * r + kk)) & 1) * ((mb >> (4 * kk + c)) & 1)
                        for r in range(4) for kk in range(4) for c in range(4))
                pairs += 1
                nz += u > 0
                useful += u
    assert w == {"pairs": pairs, "pairs_nonzero": nz, "flops_useful": 2 * useful, "flops_block": 128 * nz}
