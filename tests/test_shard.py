"""Sharding of the batched workload over ranks (CPU: gloo, world size 2).

The problems are independent, so the ranks share no data; only the job's
time (max) and work (sum) are reduced, once per run.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from cumc3d_b200 import models, shard


def test_shard_covers_every_problem_once_and_balances_the_work():
    costs = [p["n"] ** 2 for p in models.batch_problems(512)]
    for world in (1, 2, 3, 4, 8):
        parts = [shard.shard_problems(costs, r, world) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(512))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) / (sum(loads) / world) < 1.05
    with pytest.raises(ValueError):
        shard.shard_problems(costs, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        costs = [p["n"] ** 2 for p in models.batch_problems(512)]
        mine = shard.shard_problems(costs, rank, world)
        # what every rank would run, gathered to check the partition
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        # timing and work: max of the times, sum of the zone-updates
        t = shard.max_over_ranks(1.5 + rank, dist)
        w = shard.sum_over_ranks(len(mine), dist)
        np.save(os.path.join(out_dir, "r%d.npy" % rank),
                np.array([t, w, len(sorted(i for g in gathered for i in g)),
                          len(set(i for g in gathered for i in g))]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_the_batch_and_reduce_time_and_work(tmp_path):
    world, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    for r in range(world):
        t, w, n_all, n_unique = np.load(tmp_path / ("r%d.npy" % r))
        assert t == 2.5          # max over ranks of 1.5, 2.5
        assert w == 512          # every problem counted once
        assert n_all == 512 and n_unique == 512
