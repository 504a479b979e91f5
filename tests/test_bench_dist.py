"""Host-side logic of `bench.py --gpus N` for N > 1, run as two gloo ranks on the CPU.

The GPU path uses the same functions over NCCL: one process per GPU, a barrier around the
timed region, the step time reduced as the max over ranks, whole-job throughput = the
bytes all ranks processed / that time.  The reference arm runs on rank 0 alone.
"""
import json
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, q) -> None:
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    w, r, local = bench.dist_setup(world)
    assert (w, r, local) == (world, rank, rank)
    assert dist.get_backend() == "gloo"
    bench.barrier(w)
    ms_local = 10.0 + 5.0 * rank  # rank 1 is the slow one
    ms = bench.allreduce_max(ms_local, w)
    value = bench.job_throughput(w, 2e9, ms / 1e3)
    bench.barrier(w)
    dist.destroy_process_group()
    q.put((rank, ms_local, ms, value))


def test_gloo_two_ranks_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1]
    # every rank reports the slowest rank's time and the same whole-job throughput
    assert all(o[2] == 15.0 for o in out)
    assert out[0][3] == out[1][3] == pytest.approx(2 * 2e9 / 15e-3 / 1e9)


def test_job_throughput_weak_scaling():
    sys.path.insert(0, ROOT)
    import bench
    one = bench.job_throughput(1, 4e9, 1.0)
    assert bench.job_throughput(2, 4e9, 1.0) == pytest.approx(2 * one)
    assert bench.job_throughput(8, 4e9, 2.0) == pytest.approx(4 * one)


@pytest.mark.parametrize("workload", ["sketch", "randsvd", "batched", "serve"])
def test_reference_arm_nonzero_rank_exits_without_work(workload):
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3", "--workload", workload],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_reference_arm_rank0_prints_one_line():
    """Rank 0 of a two-rank launch times the CPU restatement and prints one JSON line."""
    env = dict(os.environ, RANK="0", LOCAL_RANK="0", WORLD_SIZE="2", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3", "--rows", "65536"],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
