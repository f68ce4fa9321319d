"""Partition of independent work units over ranks (one process per GPU).

Disorder realisations and eigensolve requests are independent: ranks exchange nothing on the data path.
Each rank takes its share (balanced by estimated cost, the chi^3 scaling of the matvec times the number of
bonds, or times D and the complex factor for a single eigensolve request), runs it on its own GPU, and the host
side gathers the per-unit results with a torch.distributed object gather (any backend; gloo on CPU in the
tests). This replaces the reference's SLURM job arrays (slurm/submit_jobarray.py:49-95), which run one
realisation per process and merge files afterwards.

The runners are injectable (``runner=``): the default runs the unit on this rank's GPU through the library,
and the CPU tests pass a host computation so that the partition, the per-rank call and the gather they exercise
are exactly the ones a GPU job runs.
"""
import heapq


def realisation_cost(L, chi_max):
    """Relative cost of one fDMRG realisation: bonds x chi^3 (matvec-dominated)."""
    return float(max(L - 1, 1)) * float(chi_max) ** 3


def request_cost(chi, D, cplx):
    """Relative cost of one eigensolve request: its matvec's chi^3 D term, x4 for complex arithmetic."""
    return float(chi) ** 3 * float(D) * (4.0 if cplx else 1.0)


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


def _world_rank(dist):
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    return world, (dist.get_rank() if world > 1 else 0)


def _run_share(costs, units, runner, dist):
    """This rank's share of `units` through runner(list of units) -> (results, statuses, seconds); gathered."""
    world, rank = _world_rank(dist)
    mine = partition_by_cost(costs, world)[rank]
    local = {}
    secs = 0.0
    if mine:
        res, st, secs = runner([units[i] for i in mine])
        if len(res) != len(mine) or len(st) != len(mine):
            raise RuntimeError("runner returned a different number of results than units it was given")
        local = {i: (r, s) for i, r, s in zip(mine, res, st)}
    allr = gather_results(local, dist)
    n = len(units)
    missing = [i for i in range(n) if i not in allr]
    if missing:
        raise RuntimeError(f"units {missing[:8]} were processed by no rank")
    return [allr[i][0] for i in range(n)], [allr[i][1] for i in range(n)], secs


def ensemble_sharded(realisations, dist=None, runner=None, **kw):
    """Run this rank's share of an fDMRG ensemble (heff_ensemble_run on its own GPU) and gather all results.

    realisations: list of (h_fields, chi_max, seed) as for `dmrg_b200.ensemble`; runner: a callable with the
    signature and return value of `dmrg_b200.ensemble` (default: that function with **kw). Returns (results in
    unit order, status codes in unit order, this rank's wall seconds)."""
    if runner is None:
        from . import ensemble

        def runner(units):
            return ensemble(units, **kw)

    chi_default = kw.get("chi_max", 64)
    costs = [realisation_cost(len(h), chi or chi_default) for h, chi, _ in realisations]
    return _run_share(costs, realisations, runner, dist)


def serve_sharded(specs, dist=None, runner=None, **kw):
    """Run this rank's share of a stream of eigensolve requests on its own GPU's server and gather the answers.

    specs: list of request descriptions (dicts with at least chi, D, cplx; see `dmrg_b200.serve_specs`);
    runner: a callable taking this rank's list of specs and returning (responses, status codes, wall seconds)
    (default: `dmrg_b200.serve_specs` with **kw, its server stats dropped). Returns (responses in request order,
    status codes in request order, this rank's wall seconds)."""
    if runner is None:
        from . import serve_specs

        def runner(units):
            resp, st, secs, _ = serve_specs(units, **kw)
            return resp, st, secs

    costs = [request_cost(s["chi"], s["D"], s["cplx"]) for s in specs]
    return _run_share(costs, specs, runner, dist)
