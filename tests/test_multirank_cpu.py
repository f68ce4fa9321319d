"""Multi-rank host logic on CPU (gloo, world_size 2): the partition of independent units over ranks, the gather
of their results, the max-over-ranks timing reduction and the whole-job throughput of the bench, and the
reference arm's rank-0-only behaviour under torchrun.  No GPU: the units here are host computations."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from dmrg_b200 import shard  # noqa: E402


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_covers_every_unit_once_and_balances():
    costs = [shard.realisation_cost(L, chi) for L, chi in [(12, 32), (24, 256), (16, 64), (20, 128), (12, 256), (24, 32), (16, 128)]]
    for world in (1, 2, 3, 8):
        parts = shard.partition_by_cost(costs, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT bound: no rank exceeds the mean load by more than the largest unit
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-9
    assert shard.partition_by_cost([], 2) == [[], []]
    with pytest.raises(ValueError):
        shard.partition_by_cost([1.0], 0)


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        # the slowest rank's time is the job's time, per entry
        mx = bench.reduce_max_over_ranks([10.0 + rank, 5.0 - rank], dist)
        # each rank processes its share of the units (here: squares of the unit index) and all ranks see all results
        costs = [float(c) for c in (9, 1, 4, 7, 3, 3, 8)]
        mine = shard.partition_by_cost(costs, world)[rank]
        res = shard.gather_results({i: i * i for i in mine}, dist)
        q.put((rank, mx, mine, res))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_reduce_and_gather():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    for rank, mx, mine, res in out:
        assert mx == [11.0, 5.0]
        assert res == {i: i * i for i in range(7)}
    assert sorted(out[0][2] + out[1][2]) == list(range(7))
    assert not set(out[0][2]) & set(out[1][2])


def test_job_throughput_is_all_work_over_slowest_rank():
    import bench

    F = bench.matvec_flops(4, 1024, 1024, 3, 3, True)
    one = bench.job_tflops(F, 20, 1, 132.0)
    two = bench.job_tflops(F, 20, 2, 132.0)
    assert abs(two - 2 * one) < 1e-9 * two
    assert abs(one - F * 20 / 0.132 / 1e12) < 1e-9 * one


def test_reference_arm_non_zero_rank_exits_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
