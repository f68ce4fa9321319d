"""Partition of independent work units over ranks (one process per GPU).

Disorder realisations and eigensolve requests are independent: ranks exchange nothing on the data path.
Each rank takes its share (balanced by estimated cost, the chi^3 scaling of the matvec times the number of
bonds), runs it on its own GPU, and the host side gathers the per-unit results with a torch.distributed object
gather (any backend; gloo on CPU in the tests). This replaces the reference's SLURM job arrays
(slurm/submit_jobarray.py:49-95), which run one realisation per process and merge files afterwards.
"""
import heapq


def realisation_cost(L, chi_max):
    """Relative cost of one fDMRG realisation: bonds x chi^3 (matvec-dominated)."""
    return float(max(L - 1, 1)) * float(chi_max) ** 3


def partition_by_cost(costs, world):
    """Longest-processing-time partition of units with the given costs over `world` ranks.

    Deterministic: units are taken by decreasing cost (ties by index) and given to the least-loaded rank
    (ties by rank). Returns one ascending list of unit indices per rank; every unit appears exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def gather_results(local, dist=None):
    """Merge per-rank {unit index: result} dicts into one dict on every rank (all_gather_object)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, dict(local))
    out = {}
    for p in parts:
        for k, v in p.items():
            if k in out:
                raise RuntimeError(f"unit {k} was processed by two ranks")
            out[k] = v
    return out


def ensemble_sharded(realisations, dist=None, **kw):
    """Run this rank's share of an fDMRG ensemble (heff_ensemble_run on its own GPU) and gather all results.

    realisations: list of (h_fields, chi_max, seed) as for `dmrg_b200.ensemble`. Returns (results in unit order,
    status codes in unit order, this rank's wall seconds)."""
    from . import ensemble

    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    rank = dist.get_rank() if world > 1 else 0
    chi_default = kw.get("chi_max", 64)
    costs = [realisation_cost(len(h), chi or chi_default) for h, chi, _ in realisations]
    mine = partition_by_cost(costs, world)[rank]
    local = {}
    secs = 0.0
    if mine:
        res, st, secs = ensemble([realisations[i] for i in mine], **kw)
        local = {i: (r, s) for i, r, s in zip(mine, res, st)}
    allr = gather_results(local, dist)
    n = len(realisations)
    return [allr[i][0] for i in range(n)], [allr[i][1] for i in range(n)], secs
