"""Multi-GPU plumbing: one process per GPU, no exchange step on the data path.

Every pixel and every view of the renderer is independent, so N GPUs run N
replicas: each rank renders its own frames (weak scaling) or its own share of
a batch of views; the only collective is the max over ranks of the measured
times.  These helpers hold that logic so it is tested on CPU with gloo.
"""


def shard_views(views, rank, world):
    """The views rank `rank` of `world` renders: every world-th view, so each
    rank gets a similar mix of resolutions and metric families."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    return list(views[rank::world])


def frame_times_for_rank(times, rank):
    """Animation times of a rank's replica: the workload's frame times shifted
    by the rank, so replicas render distinct frames of the same workload."""
    return [t + float(rank) for t in times]


def max_over_ranks(values, world, device=None):
    """Element-wise max of a list of floats over all ranks (one all_reduce;
    values unchanged on a single process)."""
    if world <= 1:
        return list(values)
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()
