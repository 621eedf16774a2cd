"""The multi-process host path on CPU: two gloo ranks, as bench.py and a
batched sweep run them one process per GPU.

One simulation does not shard (every step is a chain of whole-grid solves),
so each rank runs an independent replica or its own share of a sweep of
independent simulations; the only cross-rank traffic is the timing: a
barrier before the timed region and the maximum of the ranks' durations."""
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    import datetime
    import json

    import torch.distributed as dist

    import bench
    import vdropimpact_b200 as V

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        cfgs = V.sweep_configs(40, seed=5)
        mine = V.shard_sweep(cfgs, rank, world)
        shards = [None] * world
        dist.all_gather_object(shards, mine)
        cost = sum(V.sweep_cost(cfgs[k]) for k in mine)
        costs = [None] * world
        dist.all_gather_object(costs, cost)
        bench.barrier(world)
        t = bench.dist_max(10.0 * (rank + 1), world)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"shards": shards, "costs": costs, "max": t, "mine": mine}, f)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_a_sweep_and_time_by_the_slowest(tmp_path):
    import json

    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    shards = res[0]["shards"]
    # every rank computed the same assignment, and it covers the sweep once
    assert all(r["shards"] == shards for r in res)
    assert [r["mine"] for r in res] == shards
    flat = sorted(k for s in shards for k in s)
    assert flat == list(range(40))
    # the longest-first assignment balances the work within the largest job
    import vdropimpact_b200 as V
    cfgs = V.sweep_configs(40, seed=5)
    biggest = max(V.sweep_cost(c) for c in cfgs)
    costs = res[0]["costs"]
    assert max(costs) - min(costs) <= biggest
    # the timed region is the slowest rank's
    assert all(r["max"] == 20.0 for r in res)


def test_shard_sweep_single_rank_and_bad_rank():
    import vdropimpact_b200 as V
    cfgs = V.sweep_configs(7, seed=1)
    assert V.shard_sweep(cfgs, 0, 1) == list(range(7))
    with pytest.raises(ValueError):
        V.shard_sweep(cfgs, 2, 2)


def test_sweep_cost_is_cells_times_the_references_timesteps():
    """sweep_cost counts the timesteps fluid_2d::solve takes
    (fluid_2d.hh:82-86, fluid_2d.cc:42), as the oracle restates them."""
    sys.path.insert(0, ROOT)
    from oracle import vdi_oracle as vo
    import vdropimpact_b200 as V
    for cfg in V.sweep_configs(12, seed=9):
        p = vo.parse_cfg(cfg)
        l, _ = p.timestep_select(p.t_end / p.nframes)
        assert V.sweep_cost(cfg) == float(p.m * p.n * l * p.nframes)
