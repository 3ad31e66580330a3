"""The ensemble sharded over two ranks, with the product's own Ensemble path.

Two gloo ranks (spawned processes) split a ragged batch of four-quadrant
problems with the cost-balanced partition and each steps its share in one
persistent ensemble launch on this box's GPU.  The ranks take turns on the
GPU (a gloo barrier between them), so no two processes' kernels run at the
same time and no kernel waits on another rank.  The summed objective (the
final total energies) must equal a single-rank run of the whole batch: every
problem's result is bit-equal whatever batch it rides in, so the sums differ
only in the order of the final additions."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from test_sharding import free_port

pytestmark = pytest.mark.gpu

SIDES = [(64, 96), (128, 128), (100, 37), (200, 64), (48, 48), (256, 90), (90, 150), (30, 200)]
KW = dict(gamma=1.4, limiter="Minmod", riemann="HLLC", bc=["NullGradient"] * 4)
NSTEPS = 20


def configs():
    return [dict(nx=list(s), **KW) for s in SIDES]


def set_initial(p, dom):
    from heraclespp_b200 import setups

    dom.set_state_from_prim(*setups.four_quadrant(setups.Grid.from_domain(dom), seed=500 + p))


def _worker(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist

    from heraclespp_b200.sharding import _ensemble_runner, run_sharded, torch_reducers

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        inner = _ensemble_runner(NSTEPS, set_initial, strip_rows=64)

        def in_turn(my_configs, my_indices):
            out = None
            for turn in range(world):
                if turn == rank:
                    out = inner(my_configs, my_indices)
                dist.barrier()
            return out

        rs, rm = torch_reducers()
        res = run_sharded(configs(), NSTEPS, rank=rank, world=world, set_initial=set_initial, runner=in_turn,
                          reduce_sum=rs, reduce_max=rm)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(repr((res["indices"], res["objective_part"], res["objective"])))
    finally:
        dist.destroy_process_group()


def test_two_ranks_run_the_ensemble_and_match_one_rank(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    results = [eval((tmp_path / f"rank{r}.txt").read_text()) for r in range(world)]
    assert sorted(i for r in results for i in r[0]) == list(range(len(SIDES)))
    assert all(len(r[0]) > 0 for r in results)

    from heraclespp_b200.sharding import run_sharded

    one = run_sharded(configs(), NSTEPS, rank=0, world=1, set_initial=set_initial, strip_rows=64)
    for r in results:
        assert r[2] == pytest.approx(one["objective"], rel=1e-13, abs=0)
    assert sum(r[1] for r in results) == pytest.approx(one["objective"], rel=1e-13, abs=0)
    assert np.isfinite(one["objective"]) and one["objective"] > 0
