"""Sharding the batched ensemble over ranks (one process per GPU).

The problems of an ensemble are independent, so the unit that shards is the
problem: each rank steps its own subset in one persistent launch
(``Ensemble.run``) and the only exchange is the final sum of the objective
(the total energies of the final states) plus, for the timing, the maximum of
the ranks' device times.  There is no per-step collective.

The assignment is longest-processing-time greedy on cells x steps, which
keeps the largest rank load within 4/3 of the optimum.
"""
from __future__ import annotations

from typing import Callable, Sequence


def problem_cost(nx: Sequence[int], nsteps: int = 1) -> int:
    """Work of one problem: interior cells x steps."""
    cells = 1
    for n in nx:
        cells *= int(n)
    return cells * int(nsteps)


def partition(costs: Sequence[float], world: int) -> list[list[int]]:
    """Assigns problem indices to ranks: by decreasing cost (ties by index),
    each to the currently lightest rank (ties by rank).  Deterministic; every
    rank computes the same answer.  Returns each rank's indices, ascending."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    share: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        share[r].append(i)
        load[r] += float(costs[i])
    return [sorted(s) for s in share]


def loads(costs: Sequence[float], share: Sequence[Sequence[int]]) -> list[float]:
    return [sum(float(costs[i]) for i in s) for s in share]


def total_energy(domain) -> float:
    """Sum of E dV over the interior of one problem (compensated FP64 sum on
    the device, hcl_conservation_sums)."""
    return float(domain.conservation_sums()[domain.ndim + 1])


def run_sharded(configs: Sequence[dict], nsteps: int, *, rank: int, world: int, set_initial: Callable,
                runner: Callable | None = None, reduce_sum: Callable | None = None, reduce_max: Callable | None = None,
                **run_kw):
    """Runs this rank's share of the ensemble and combines the objective.

    configs      keyword dicts of every problem (``nx`` plus the physics keys)
    set_initial  set_initial(p, domain) sets problem p's initial state
    runner       runner(my_configs, my_indices) -> (objective_part, seconds);
                 default: one Ensemble over this rank's problems
    reduce_sum / reduce_max: the cross-rank reductions (torch.distributed
                 all_reduce in practice); identity when world == 1
    Returns a dict with the rank's indices, its objective part and time, the
    summed objective and the maximum time over ranks."""
    costs = [problem_cost(c["nx"], nsteps) for c in configs]
    share = partition(costs, world)
    mine = share[rank]
    if runner is None:
        runner = _ensemble_runner(nsteps, set_initial, **run_kw)
    part, seconds = runner([configs[i] for i in mine], mine)
    total = reduce_sum(part) if reduce_sum is not None else part
    slowest = reduce_max(seconds) if reduce_max is not None else seconds
    return {"indices": mine, "objective_part": part, "seconds": seconds, "objective": total,
            "max_seconds": slowest, "loads": loads(costs, share)}


def _ensemble_runner(nsteps: int, set_initial: Callable, **run_kw):
    def run(my_configs, my_indices):
        import time

        import torch

        from . import Ensemble

        if not my_configs:
            return 0.0, 0.0
        ens = Ensemble(my_configs)
        for d, p in zip(ens.domains, my_indices):
            set_initial(p, d)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ens.run(nsteps, **run_kw)
        torch.cuda.synchronize()
        seconds = time.perf_counter() - t0
        part = sum(total_energy(d) for d in ens.domains)
        ens.close()
        return part, seconds

    return run


def torch_reducers(device=None):
    """all_reduce-based reduce_sum / reduce_max over the default process group
    (gloo on CPU tensors, NCCL on CUDA tensors)."""
    import torch
    import torch.distributed as dist

    def red(x, op):
        t = torch.tensor([float(x)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=op)
        return float(t.item())

    return (lambda x: red(x, dist.ReduceOp.SUM)), (lambda x: red(x, dist.ReduceOp.MAX))
