"""CPU: the N-GPU benchmark path runs N independent replicas, one process per GPU,
with no collective on the data path; the only collective is the MAX over the ranks'
timings.  Exercised here with world size 2 on the gloo backend: every rank gets the
slowest rank's time and the whole-job rate counts both ranks' units; the reference
arm's non-zero ranks exit at once without output."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from hpgem_b200 import replicas

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seconds = 1.0 + rank  # rank 1 is the slow one
        rate, slowest = replicas.aggregate_rate(1000, seconds, world, dist)
        out.put((rank, rate, slowest, replicas.max_over_ranks(10.0 * (world - rank), dist)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rate_with_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, rate, slowest, m in res:
        assert slowest == 2.0  # the slowest rank's time, on every rank
        assert rate == 1000 * 2 / 2.0
        assert m == 20.0


def test_single_process_needs_no_group():
    from hpgem_b200 import replicas

    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.aggregate_rate(100, 2.0, 1) == (50.0, 2.0)


def test_reference_arm_non_zero_rank_exits_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
