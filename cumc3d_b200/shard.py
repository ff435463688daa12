"""Multi-GPU plumbing for the workloads that shard.

The 3D grid path runs as independent replicas (one per GPU) until the halo
exchange exists; the batched 1D workload shards for real: its problems are
independent, so each rank takes a share of them and no collective touches
the data path.  Only the timing and the zone-update count cross ranks
(max of the device time, sum of the work), once per run.
"""
import os


def dist_env():
    """(world, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard_problems(costs, rank, world):
    """Indices of the problems rank `rank` runs: largest cost first, dealt in
    a snake order (0,1,..,w-1,w-1,..,0,...) so every rank gets a similar
    total.  Every index appears on exactly one rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    mine = []
    for pos, i in enumerate(order):
        lap, r = divmod(pos, world)
        owner = r if lap % 2 == 0 else world - 1 - r
        if owner == rank:
            mine.append(i)
    return sorted(mine)


def max_over_ranks(x, dist, device="cpu"):
    """The maximum of a float over all ranks (the job's time)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, dist, device="cpu"):
    """The sum of a number over all ranks (the job's work)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
