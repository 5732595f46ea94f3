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


def orbit_frames_for_rank(n_orbit, per_rank, rank):
    """Frame indices of a rank's replica of an orbit workload: `per_rank` frames
    evenly spaced over the `n_orbit`-frame orbit, offset by the rank, so up to
    n_orbit / per_rank ranks render distinct frames of equal cost on average."""
    if per_rank < 1 or n_orbit < per_rank or rank < 0:
        raise ValueError("bad orbit sharding")
    stride = n_orbit // per_rank
    return [(j * stride + rank) % n_orbit for j in range(per_rank)]


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
