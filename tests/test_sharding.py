"""Sharding the ensemble's problems over ranks (CPU): the assignment, and the
cross-rank combination of the objective and the timing over a 2-rank gloo
group with a stand-in runner (no GPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from heraclespp_b200.sharding import loads, partition, problem_cost, run_sharded

SIDES = (128, 256, 512, 1024)


def bench_sizes(n=96, seed=2024):
    rng = np.random.default_rng(seed)
    return [(int(rng.choice(SIDES)), int(rng.choice(SIDES))) for _ in range(n)]


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_partition_covers_every_problem_once_and_balances(world):
    costs = [problem_cost(nx, 300) for nx in bench_sizes()]
    share = partition(costs, world)
    assert len(share) == world
    flat = sorted(i for s in share for i in s)
    assert flat == list(range(len(costs)))
    ld = loads(costs, share)
    # longest-processing-time bound: makespan <= 4/3 of the optimum's lower bound
    lower = max(sum(costs) / world, max(costs))
    assert max(ld) <= 4.0 / 3.0 * lower
    assert partition(costs, world) == share  # deterministic


def test_partition_edge_cases():
    assert partition([], 3) == [[], [], []]
    assert partition([5.0], 2) == [[0], []]
    assert partition([1, 1, 1, 1], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        partition([1.0], 0)


def fake_runner(my_configs, my_indices):
    # objective part: a value per problem; "time": its cost
    part = sum(1000.0 + i for i in my_indices)
    seconds = sum(problem_cost(c["nx"], 1) for c in my_configs) * 1e-9
    return part, seconds


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist

    from heraclespp_b200.sharding import torch_reducers

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        configs = [dict(nx=list(nx)) for nx in bench_sizes(24, seed=7)]
        rs, rm = torch_reducers()
        res = run_sharded(configs, 10, rank=rank, world=world, set_initial=None, runner=fake_runner, reduce_sum=rs,
                          reduce_max=rm)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(repr((res["indices"], res["objective"], res["max_seconds"], res["seconds"])))
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_objective_and_timing_over_gloo(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    results = [eval((tmp_path / f"rank{r}.txt").read_text()) for r in range(world)]
    configs = [dict(nx=list(nx)) for nx in bench_sizes(24, seed=7)]
    idx = sorted(i for r in results for i in r[0])
    assert idx == list(range(len(configs)))
    expect_total = sum(1000.0 + i for i in range(len(configs)))
    for r in results:
        assert r[1] == pytest.approx(expect_total, rel=0, abs=1e-9)
        assert r[2] == max(x[3] for x in results)
