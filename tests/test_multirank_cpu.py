"""Multi-rank host logic on CPU (gloo, world_size 2): the partition of independent units over ranks, the gather
of their results, the max-over-ranks timing reduction and the whole-job throughput of the bench, and the
reference arm's rank-0-only behaviour under torchrun.  No GPU: the units here are host computations.

The sharded ensemble and the sharded serving stream run through `shard.ensemble_sharded` and
`shard.serve_sharded` themselves, with host stand-ins injected for the per-GPU runners (the free-fermion
ground energy of each realisation; the lowest eigenvalue of a small seeded Hermitian matrix per request), so
the partition, the per-rank call and the gather are the code a multi-GPU job runs."""
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


def _ff_runner(units):
    """Host stand-in for dmrg_b200.ensemble: the exact ground energy of each realisation (free fermions)."""
    from oracle import physics as ph

    res = [{"energy": ph.free_fermion_ground(h), "L": len(h), "chi_max": chi, "seed": seed} for h, chi, seed in units]
    return res, [0] * len(units), 0.01


def _eig_runner(units):
    """Host stand-in for dmrg_b200.serve_specs: the lowest eigenvalue of a seeded Hermitian matrix per request."""
    import numpy as np

    out = []
    for sp in units:
        rng = np.random.default_rng(sp["seed"])
        n = 4 * sp["D"]
        X = rng.standard_normal((n, n)) + (1j * rng.standard_normal((n, n)) if sp["cplx"] else 0)
        out.append({"eigval": float(np.linalg.eigvalsh((X + X.conj().T) / 2)[0]), "id": sp["seed"]})
    return out, [0] * len(units), 0.02


def _realisations():
    from oracle import physics as ph

    Ls, chis = [12, 16, 20, 24, 12, 16, 20], [32, 256, 64, 128, 256, 32, 64]
    return [(ph.random_fields(100 + i, L), chi, i) for i, (L, chi) in enumerate(zip(Ls, chis))]


def _specs():
    chis, Ds = [64, 2048, 300, 1024, 128, 700, 90, 512, 64], [3, 9, 3, 3, 9, 9, 3, 9, 3]
    return [{"chi": c, "D": D, "cplx": i % 3 == 1, "seed": 1000 + i} for i, (c, D) in enumerate(zip(chis, Ds))]


def _shard_worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ens, ens_st, _ = shard.ensemble_sharded(_realisations(), dist, runner=_ff_runner)
        srv, srv_st, _ = shard.serve_sharded(_specs(), dist, runner=_eig_runner)
        reals = _realisations()
        costs = [shard.realisation_cost(len(h), c) for h, c, _ in reals]
        mine_ens = shard.partition_by_cost(costs, world)[rank]
        costs_s = [shard.request_cost(s["chi"], s["D"], s["cplx"]) for s in _specs()]
        mine_srv = shard.partition_by_cost(costs_s, world)[rank]
        q.put((rank, ens, ens_st, srv, srv_st, mine_ens, mine_srv))
    finally:
        dist.destroy_process_group()


def _run_world(target, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(out, key=lambda t: t[0])


def test_sharded_ensemble_and_serving_gather_every_unit_in_order():
    out = _run_world(_shard_worker)
    ens1, _, _ = _ff_runner(_realisations())
    srv1, _, _ = _eig_runner(_specs())
    for rank, ens, ens_st, srv, srv_st, _, _ in out:
        # every rank holds every unit's result, in unit order, equal to the one-process run
        assert ens == ens1 and ens_st == [0] * len(ens1)
        assert srv == srv1 and srv_st == [0] * len(srv1)
    # the two ranks did disjoint shares that cover all units, and the cost balance puts the two largest requests apart
    assert sorted(out[0][5] + out[1][5]) == list(range(len(ens1))) and not set(out[0][5]) & set(out[1][5])
    assert sorted(out[0][6] + out[1][6]) == list(range(len(srv1))) and not set(out[0][6]) & set(out[1][6])
    big = sorted(range(len(srv1)), key=lambda i: -shard.request_cost(_specs()[i]["chi"], _specs()[i]["D"], _specs()[i]["cplx"]))[:2]
    assert (big[0] in out[0][6]) != (big[1] in out[0][6])


def test_sharded_runner_must_answer_every_unit():
    def short(units):
        return [0] * (len(units) - 1), [0] * (len(units) - 1), 0.0

    with pytest.raises(RuntimeError):
        shard.serve_sharded(_specs(), None, runner=short)
    one, st, _ = shard.ensemble_sharded(_realisations(), None, runner=_ff_runner)
    assert one == _ff_runner(_realisations())[0]


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
